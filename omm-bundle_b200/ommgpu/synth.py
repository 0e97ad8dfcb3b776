"""Seeded synthetic inputs for the libOMM workloads (no dataset or checkpoint is involved).

Five workloads, named by what they are:

* ``dense_832``      real dense m=832, n=128 with a constructed spectrum
  (S = L L^T, H = L Q diag(lam) Q^T L^T), FP64, the CPU-runnable case.
* ``lattice_8x8x8``  512 atoms on a periodic 8x8x8 simple-cubic lattice x 24
  orbitals -> m=12,288, n=1,536, H/S stored as CSC with 24x24 blocks for atom
  pairs within two lattice spacings (33 neighbours incl. self, 6.4 % fill).
* ``lattice_16x8x8`` the same generator at 1,024 atoms: m=24,576, n=3,072.
* ``zdense_4096``    complex Hermitian dense m=4,096, n=512 built like
  ``dense_832`` with a unitary Q, plus 16 Hermitian sparse perturbations V_k
  (2 % fill, entries N(0, 0.01)) for H(theta) = H0 + sum_k theta_k V_k.
* ``lattice_16x16x8`` the generator at 2,048 atoms: m=49,152, n=6,144 plus 8
  sparse perturbations V_k.

Lattice H blocks are exp(-r) x Gaussian and S blocks exp(-r^2) x Gaussian
(symmetric pairs, S onsite = I).  The onsite H block is a Gaussian plus a level
splitting (3 levels at -1, 21 at +1 per atom) so that the spectrum has a gap at
n = 3 x atoms; OMM minimises the Kim functional, whose minimum is the
occupied subspace only when the system is gapped.  H is then shifted by
mu = (lam_n + lam_{n+1}) / 2 of the generalized problem (H - mu S), so exactly
n eigenvalues are negative.  mu comes from a dense FP64 eigensolve; results
for the named workloads are cached in ``spectra.json`` beside this file.

All arrays are column-major (Fortran order) like the reference's matrices.
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SPECTRA = os.path.join(_HERE, "spectra.json")
DEFAULT_SEED = 123456

# generator constants of the lattice workloads
NORB = 24
NOCC = 3
S_SCALE = 0.04  # off-site S block = S_SCALE * exp(-r^2) * N(0,1)
H_SCALE = 0.06  # off-site H block = H_SCALE * exp(-r) * N(0,1)
ONSITE_SCALE = 0.10  # onsite H block = levels + ONSITE_SCALE * sym(N(0,1))
LEVEL_OCC, LEVEL_VIR = -1.0, 1.0


@dataclass
class CSCMatrix:
    """Square or rectangular CSC with 0-based offsets and rows (values float64 / complex128)."""

    dim1: int
    dim2: int
    colptr: np.ndarray
    rowind: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.colptr[-1])

    def to_dense(self) -> np.ndarray:
        out = np.zeros((self.dim1, self.dim2), dtype=self.val.dtype, order="F")
        cols = np.repeat(np.arange(self.dim2), np.diff(self.colptr))
        out[self.rowind, cols] = self.val
        return out

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.val, self.rowind, self.colptr), shape=(self.dim1, self.dim2))

    @staticmethod
    def from_scipy(a) -> "CSCMatrix":
        a = a.tocsc()
        a.sort_indices()
        return CSCMatrix(a.shape[0], a.shape[1], a.indptr.astype(np.int32), a.indices.astype(np.int32),
                         np.ascontiguousarray(a.data))

    def nbytes(self, val_bytes: int) -> int:
        return self.nnz * (val_bytes + 4) + (self.dim2 + 1) * 4


@dataclass
class Problem:
    name: str
    m: int
    n: int
    H: object  # np.ndarray (dense, Fortran order) or CSCMatrix
    S: object
    mu: float = 0.0
    e_exact: float | None = None  # sum of the n lowest eigenvalues of (H - mu S, S)
    V: list = field(default_factory=list)  # sparse perturbations (CSCMatrix)
    meta: dict = field(default_factory=dict)

    @property
    def is_real(self) -> bool:
        v = self.H.val if isinstance(self.H, CSCMatrix) else self.H
        return np.isrealobj(v)


# --------------------------------------------------------------------------
# lattice generator
# --------------------------------------------------------------------------
def _shell():
    d = [(x, y, z) for x in range(-2, 3) for y in range(-2, 3) for z in range(-2, 3) if x * x + y * y + z * z <= 4]
    return np.array(d, dtype=np.int64)


def lattice_blocks(L, seed: int = DEFAULT_SEED, norb: int = NORB, nocc: int = NOCC):
    """Block lists of the lattice H and S: (pairs (I,J) with I<=J, H blocks, S blocks, distances)."""
    Lx, Ly, Lz = L
    if min(L) < 5:
        raise ValueError("lattice sides must be >= 5 so that the 2-spacing shells do not wrap onto themselves")
    rng = np.random.default_rng(seed)
    na = Lx * Ly * Lz
    d = _shell()
    a = np.arange(na)
    x, y, z = a // (Ly * Lz), (a // Lz) % Ly, a % Lz
    # neighbour b of atom a for each shell vector
    bx = (x[:, None] + d[None, :, 0]) % Lx
    by = (y[:, None] + d[None, :, 1]) % Ly
    bz = (z[:, None] + d[None, :, 2]) % Lz
    b = (bx * Ly + by) * Lz + bz
    r = np.sqrt((d * d).sum(1)).astype(np.float64)
    I = np.repeat(a, len(d))
    J = b.reshape(-1)
    R = np.tile(r, na)
    keep = I <= J
    I, J, R = I[keep], J[keep], R[keep]
    order = np.lexsort((J, I))
    I, J, R = I[order], J[order], R[order]
    npair = len(I)
    G = rng.standard_normal((npair, norb, norb))
    G2 = rng.standard_normal((npair, norb, norb))
    onsite = I == J
    levels = np.full(norb, LEVEL_VIR)
    levels[:nocc] = LEVEL_OCC
    Hb = H_SCALE * np.exp(-R)[:, None, None] * G
    Sb = S_SCALE * np.exp(-R * R)[:, None, None] * G2
    Gs = 0.5 * (G[onsite] + np.transpose(G[onsite], (0, 2, 1)))
    Hb[onsite] = np.diag(levels)[None] + ONSITE_SCALE * Gs
    Sb[onsite] = np.eye(norb)[None]
    return I, J, Hb, Sb, na


def _blocks_to_csc(I, J, blocks, na, norb):
    """Assemble symmetric block lists (I<=J) into a full CSC with sorted rows."""
    offd = I != J
    # full list of (block row, block col, block) including transposes
    BI = np.concatenate([I, J[offd]])
    BJ = np.concatenate([J, I[offd]])
    BV = np.concatenate([blocks, np.transpose(blocks[offd], (0, 2, 1))])
    order = np.lexsort((BI, BJ))  # by block column, then block row
    BI, BJ, BV = BI[order], BJ[order], BV[order]
    nb_per_col = np.bincount(BJ, minlength=na)
    # values: for block column J, column c in 0..norb-1: concatenate block rows' column c
    m = na * norb
    colptr = np.zeros(m + 1, dtype=np.int64)
    per_col = np.repeat(nb_per_col * norb, norb)
    colptr[1:] = np.cumsum(per_col)
    nnz = int(colptr[-1])
    rowind = np.empty(nnz, dtype=np.int32)
    val = np.empty(nnz, dtype=blocks.dtype)
    starts = np.concatenate([[0], np.cumsum(nb_per_col)])
    for Jb in range(na):
        s, e = starts[Jb], starts[Jb + 1]
        rows = (BI[s:e, None] * norb + np.arange(norb)[None, :]).reshape(-1)  # (nb*norb)
        vals = BV[s:e]  # nb x norb(rows) x norb(cols)
        # column c of the block column: stack vals[:, :, c] over blocks
        cols_vals = np.transpose(vals, (2, 0, 1)).reshape(norb, -1)  # c, (block, row)
        base = colptr[Jb * norb]
        k = len(rows)
        for c in range(norb):
            rowind[base + c * k : base + (c + 1) * k] = rows
            val[base + c * k : base + (c + 1) * k] = cols_vals[c]
    return CSCMatrix(m, m, colptr.astype(np.int32), rowind, val)


def _load_spectra() -> dict:
    if os.path.exists(_SPECTRA):
        with open(_SPECTRA) as f:
            return json.load(f)
    return {}


def spectrum_key(name: str, seed: int) -> str:
    return "%s/seed=%d" % (name, seed)


def csc_device_index(A: CSCMatrix, device):
    """(rows, cols, vals) torch tensors of a CSC's nonzeros on `device`."""
    import torch

    cols = torch.repeat_interleave(torch.arange(A.dim2, device=device),
                                   torch.from_numpy(np.diff(A.colptr).astype(np.int64)).to(device))
    rows = torch.from_numpy(A.rowind.astype(np.int64)).to(device)
    return rows, cols, torch.from_numpy(np.ascontiguousarray(A.val)).to(device)


def _dense_on_device(A, device):
    """Dense torch copy (row-major [row, col]) of a CSCMatrix or ndarray on `device`; a CSC is
    expanded on the device (no dense host copy: at m = 49,152 one dense FP64 matrix is 19.3 GB)."""
    import torch

    if not isinstance(A, CSCMatrix):
        return torch.from_numpy(np.ascontiguousarray(A)).to(device)
    dt = torch.complex128 if np.iscomplexobj(A.val) else torch.float64
    out = torch.zeros(A.dim1, A.dim2, dtype=dt, device=device)
    rows, cols, vals = csc_device_index(A, device)
    out[rows, cols] = vals
    return out


def generalized_eigvals(H, S, device: str | None = None) -> np.ndarray:
    """All eigenvalues of H x = lam S x in FP64 (dense; torch on CUDA when available, else SciPy)."""
    try:
        import torch

        if device is None:
            device = "cuda" if torch.cuda.is_available() else "cpu"
        if device == "cuda":
            Ht = _dense_on_device(H, device)
            St = _dense_on_device(S, device)
            Lc = torch.linalg.cholesky(St)
            del St
            A = torch.linalg.solve_triangular(Lc, Ht, upper=False)
            del Ht
            A = torch.linalg.solve_triangular(Lc, A.mH, upper=False)  # L^-1 H L^-H (Hermitian)
            del Lc
            try:
                w = torch.linalg.eigvalsh(A).cpu().numpy()
            except RuntimeError:
                # cuSOLVER's syevd rejects very large orders (its workspace query fails at
                # m = 49,152): LAPACK on the host instead
                Ah = A.cpu()
                A = None
                torch.cuda.empty_cache()
                w = torch.linalg.eigvalsh(Ah).numpy()
            A = None
            torch.cuda.empty_cache()
            return w
    except ImportError:
        pass
    import scipy.linalg as sl

    Hd = H.to_dense() if isinstance(H, CSCMatrix) else H
    Sd = S.to_dense() if isinstance(S, CSCMatrix) else S
    return sl.eigh(Hd, Sd, eigvals_only=True, driver="gvd")


def lattice(L, seed: int = DEFAULT_SEED, name: str | None = None, norb: int = NORB, nocc: int = NOCC,
            nperturb: int = 0, compute_mu: bool = True) -> Problem:
    I, J, Hb, Sb, na = lattice_blocks(L, seed, norb, nocc)
    H = _blocks_to_csc(I, J, Hb, na, norb)
    S = _blocks_to_csc(I, J, Sb, na, norb)
    m, n = na * norb, na * nocc
    name = name or "lattice_%dx%dx%d" % tuple(L)
    prob = Problem(name, m, n, H, S, meta={"atoms": na, "norb": norb, "nocc": nocc, "seed": seed,
                                           "nnz": H.nnz, "fill": H.nnz / float(m * m), "block": norb})
    if compute_mu:
        _apply_mu(prob, seed)
    if nperturb:
        prob.V = sparse_perturbations(m, nperturb, fill=0.02 if m <= 8192 else 32.0 / m, seed=seed + 7,
                                      complex_=False)
    return prob


def _apply_mu(prob: Problem, seed: int):
    key = spectrum_key(prob.name, seed)
    cache = _load_spectra()
    if key in cache:
        mu, e_exact = cache[key]["mu"], cache[key]["e_exact"]
    else:
        w = generalized_eigvals(prob.H, prob.S)
        n = prob.n
        mu = 0.5 * (w[n - 1] + w[n])
        e_exact = float(np.sum(w[:n] - mu))
        prob.meta["gap"] = float(w[n] - w[n - 1])
        prob.meta["spectrum"] = [float(w[0]), float(w[n - 1]), float(w[n]), float(w[-1])]
    # H <- H - mu S on the union pattern (S and H share the block pattern)
    H, S = prob.H, prob.S
    assert np.array_equal(H.colptr, S.colptr) and np.array_equal(H.rowind, S.rowind)
    H.val = H.val - mu * S.val
    prob.mu = float(mu)
    prob.e_exact = float(e_exact)


def sparse_perturbations(m: int, count: int, fill: float, seed: int, complex_: bool, scale: float = 0.1):
    """count Hermitian sparse matrices with ~fill density and N(0, scale^2) entries."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        k = max(1, int(fill * m * m / 2))
        r = rng.integers(0, m, size=k)
        c = rng.integers(0, m, size=k)
        v = rng.standard_normal(k) * scale
        if complex_:
            v = v + 1j * rng.standard_normal(k) * scale
            v = np.where(r == c, v.real + 0j, v)
        A = sp.coo_matrix((v, (r, c)), shape=(m, m)).tocsc()
        A = A + A.conj().T
        A = A.tocsc()
        A.sum_duplicates()
        out.append(CSCMatrix.from_scipy(A))
    return out


# --------------------------------------------------------------------------
# dense generator with a constructed spectrum
# --------------------------------------------------------------------------
def dense(m: int, n: int, seed: int = DEFAULT_SEED, complex_: bool = False, name: str | None = None,
          nperturb: int = 0) -> Problem:
    rng = np.random.default_rng(seed)
    G = rng.standard_normal((m, m))
    Sm = np.eye(m) + 0.05 * 0.5 * (G + G.T)
    w, V = np.linalg.eigh(Sm)
    Sm = (V * np.clip(w, 0.8, 1.2)) @ V.T
    Sm = 0.5 * (Sm + Sm.T)
    Lc = np.linalg.cholesky(Sm)
    if complex_:
        Z = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    else:
        Z = rng.standard_normal((m, m))
    Q, R = np.linalg.qr(Z)
    Q = Q * (np.diag(R) / np.abs(np.diag(R)))[None, :]
    lam = np.concatenate([rng.uniform(-2.0, -0.5, n), rng.uniform(0.1, 3.0, m - n)])
    LQ = Lc @ Q
    Hm = (LQ * lam[None, :]) @ LQ.conj().T
    Hm = 0.5 * (Hm + Hm.conj().T)
    dt = np.complex128 if complex_ else np.float64
    H = np.asfortranarray(Hm.astype(dt))
    S = np.asfortranarray(Sm.astype(dt))
    name = name or ("zdense_%d" % m if complex_ else "dense_%d" % m)
    prob = Problem(name, m, n, H, S, mu=0.0, e_exact=float(np.sort(lam)[:n].sum()),
                   meta={"seed": seed, "lam_n": float(np.sort(lam)[n - 1]), "lam_n1": float(np.sort(lam)[n])})
    if nperturb:
        prob.V = sparse_perturbations(m, nperturb, fill=0.02, seed=seed + 11, complex_=complex_)
    return prob


WORKLOADS = {
    "dense_832": dict(kind="dense", m=832, n=128),
    "lattice_8x8x8": dict(kind="lattice", L=(8, 8, 8)),
    "lattice_16x8x8": dict(kind="lattice", L=(16, 8, 8)),
    "zdense_4096": dict(kind="zdense", m=4096, n=512, nperturb=16),
    "lattice_16x16x8": dict(kind="lattice", L=(16, 16, 8), nperturb=8),
}


def workload(name: str, seed: int = DEFAULT_SEED) -> Problem:
    w = WORKLOADS[name]
    if w["kind"] == "dense":
        return dense(w["m"], w["n"], seed, False, name)
    if w["kind"] == "zdense":
        return dense(w["m"], w["n"], seed, True, name, nperturb=w.get("nperturb", 0))
    return lattice(w["L"], seed, name, nperturb=w.get("nperturb", 0))


def lcg_c0(n: int, m: int, complex_: bool = False) -> np.ndarray:
    """C0 exactly as the reference fills it under NORAND (omm.F90:329-342, omm_rand.F90:19-55).

    x <- (1103515245 x + 12345) mod 2^31 from seed 123456, two draws per element,
    element C(j,i) = sign(0.5 r1, r2 - 0.5) in column-major order, then C *= 1e-2/sqrt(m).
    """
    cnt = 2 * n * m
    xs = np.empty(cnt, dtype=np.int64)
    x = 123456
    a, c, mod = 1103515245, 12345, 1 << 31
    # vectorised LCG by blocks: x_{k+1} = a x_k + c; use jump-ahead in chunks of 2^16
    chunk = 1 << 16
    # precompute a^k and c*(a^k-1)/(a-1) mod 2^31 for k=1..chunk
    ak = np.empty(chunk, dtype=np.int64)
    ck = np.empty(chunk, dtype=np.int64)
    pa, pc = 1, 0
    for k in range(chunk):
        pa = (pa * a) % mod
        pc = (pc * a + c) % mod
        ak[k], ck[k] = pa, pc
    pos = 0
    while pos < cnt:
        k = min(chunk, cnt - pos)
        # x_{pos+1+t} = ak[t]*x + ck[t]  (mod 2^31), computed with 64-bit safe products
        xs[pos : pos + k] = (_mulmod(ak[:k], x, mod) + ck[:k]) % mod
        x = int(xs[pos + k - 1])
        pos += k
    r = xs.astype(np.float64) / float(mod)
    r1, r2 = r[0::2], r[1::2]
    el = np.where(r2 - 0.5 >= 0.0, np.abs(0.5 * r1), -np.abs(0.5 * r1))
    C = el.reshape((m, n)).T  # element order: i (m) outer, j (n) inner
    C = np.asfortranarray(C) * (1.0e-2 / np.sqrt(float(m)))
    return C.astype(np.complex128) if complex_ else C


def _mulmod(a: np.ndarray, x: int, mod: int) -> np.ndarray:
    # a < 2^31, x < 2^31: split x into 16-bit halves to stay inside int64
    xh, xl = x >> 16, x & 0xFFFF
    return ((a * xh % mod) * 65536 + a * xl) % mod
