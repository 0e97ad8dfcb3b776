"""FP64 GEMM on the int8 tensor cores (omm_gpu_gemm_f64) against extended-precision products.

The method rounds each row of op(A) and column of op(B) to 53 bits relative
to its largest entry (an error of at most 2^-53 max_k |a_ik| per entry), forms
their product exactly and rounds once.  So every output element must lie within
2^-52 (max_k |a_ik| sum_k |b_kj| + sum_k |a_ik| max_k |b_kj| + |c_ij|) of the
product computed in 80-bit long double; and at the solver's shapes within
1e-13 sum_k |a_ik b_kj| of cuBLAS's DGEMM (whose own error is of that order)."""
import ctypes as ct

import numpy as np
import pytest

import ommgpu as G

pytestmark = pytest.mark.gpu

TOL = 2.0 ** -52


def _fn():
    L = G.lib()
    f = L.omm_gpu_gemm_f64
    f.argtypes = [ct.c_char, ct.c_char, ct.c_int, ct.c_int, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int,
                  ct.c_void_p, ct.c_int, ct.c_double, ct.c_void_p, ct.c_int]
    f.restype = ct.c_int
    L.omm_gpu_last_error.restype = ct.c_char_p
    return f, L


def _run(opA, opB, M, N, K, alpha=1.0, beta=0.0, seed=0, A=None, B=None, C0=None):
    import torch

    f, L = _fn()
    rng = np.random.default_rng(seed)
    ash = (M, K) if opA == "n" else (K, M)
    bsh = (K, N) if opB == "n" else (N, K)
    A = rng.standard_normal(ash) * np.exp(rng.uniform(-3, 3, ash)) if A is None else A
    B = rng.standard_normal(bsh) * np.exp(rng.uniform(-3, 3, bsh)) if B is None else B
    C0 = rng.standard_normal((M, N)) if C0 is None else C0
    # column-major device copies: a torch tensor of shape (cols, rows) row-major is the column-major matrix
    At = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    Bt = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    Ct = torch.from_numpy(np.ascontiguousarray(C0.T)).cuda()
    rc = f(opA.encode(), opB.encode(), M, N, K, alpha, At.data_ptr(), ash[0], Bt.data_ptr(), bsh[0], beta,
           Ct.data_ptr(), M)
    assert rc == 0, L.omm_gpu_last_error().decode()
    got = Ct.cpu().numpy().T
    opa = A if opA == "n" else A.T
    opb = B if opB == "n" else B.T
    return got, opa, opb, C0


def _exact(opa, opb, C0, alpha, beta):
    """long-double product and the normwise bound of the row/column rounding"""
    la, lb = opa.astype(np.longdouble), opb.astype(np.longdouble)
    ref = alpha * (la @ lb) + beta * C0.astype(np.longdouble)
    aa, ab = np.abs(opa), np.abs(opb)
    mag = abs(alpha) * (aa.max(axis=1)[:, None] * ab.sum(axis=0)[None, :] +
                        aa.sum(axis=1)[:, None] * ab.max(axis=0)[None, :])
    return ref, mag + np.abs(ref.astype(np.float64))


@pytest.mark.parametrize("opA", ["n", "t"])
@pytest.mark.parametrize("opB", ["n", "t"])
def test_ops_against_long_double(opA, opB):
    M, N, K = 200, 300, 777
    got, opa, opb, C0 = _run(opA, opB, M, N, K, alpha=0.75, beta=-1.25, seed=hash((opA, opB)) % 1000)
    ref, mag = _exact(opa, opb, C0, 0.75, -1.25)
    err = np.abs(got - ref.astype(np.float64))
    assert np.all(err <= TOL * mag + 1e-300), float(np.max(err / (mag + 1e-300)))


def test_ragged_tiles_and_small_k():
    for (M, N, K) in ((129, 257, 1), (1, 1, 1), (300, 17, 130), (131, 513, 4099)):
        got, opa, opb, C0 = _run("n", "n", M, N, K, seed=M + N + K)
        ref, mag = _exact(opa, opb, C0, 1.0, 0.0)
        assert np.all(np.abs(got - ref.astype(np.float64)) <= TOL * mag + 1e-300), (M, N, K)


def test_zero_rows_and_nonfinite():
    M, N, K = 160, 200, 300
    rng = np.random.default_rng(5)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    A[3, :] = 0.0          # a zero row of A: row 3 of C is exactly 0
    A[7, 11] = np.nan      # NaN in row 7: row 7 of C is NaN
    B[:, 5] = 0.0          # a zero column of B: column 5 of C is 0 (except the NaN row)
    B[20, 9] = np.inf      # Inf in column 9: column 9 is NaN
    got, opa, opb, _ = _run("n", "n", M, N, K, A=A, B=B, C0=np.zeros((M, N)))
    assert np.all(got[3, np.arange(N) != 9] == 0.0) and np.isnan(got[3, 9])  # 0 * Inf = NaN
    assert np.all(np.isnan(got[7, :]))
    assert np.all(np.isnan(got[:, 9]))
    keep = np.ones(M, bool)
    keep[7] = False
    assert np.all(got[keep, 5] == 0.0)
    clean_r = np.setdiff1d(np.arange(M), [3, 7])
    clean_c = np.setdiff1d(np.arange(N), [5, 9])
    ref, mag = _exact(opa[clean_r], opb[:, clean_c], np.zeros((len(clean_r), len(clean_c))), 1.0, 0.0)
    sub = got[np.ix_(clean_r, clean_c)]
    assert np.all(np.abs(sub - ref.astype(np.float64)) <= TOL * mag + 1e-300)


def test_solver_shape_against_cublas():
    """The Gram product's shape at lattice_8x8x8 (2n x n, K = m = 12,288) against torch's
    cuBLAS DGEMM: the two FP64 GEMMs agree within 1e-13 of |A||B|."""
    import torch

    f, L = _fn()
    g = torch.Generator(device="cuda").manual_seed(3)
    M, N, K = 3072, 1536, 12288
    X = torch.randn(K, M, generator=g, device="cuda", dtype=torch.float64) * 1e-2  # column-major M x K
    D = torch.randn(K, N, generator=g, device="cuda", dtype=torch.float64)         # column-major N x K
    out = torch.empty(N, M, device="cuda", dtype=torch.float64)
    rc = f(b"n", b"t", M, N, K, 1.0, X.data_ptr(), M, D.data_ptr(), N, 0.0, out.data_ptr(), M)
    assert rc == 0, L.omm_gpu_last_error().decode()
    ref = X.t() @ D   # (M x K) (K x N) in cuBLAS
    mag = X.t().abs() @ D.abs()
    err = ((out.t() - ref).abs() / mag).max().item()
    assert err <= 1e-13, err


def test_column_panels():
    """A residue cap small enough to split the product into column panels gives the same result."""
    import torch

    f, L = _fn()
    M, N, K = 384, 1100, 500
    try:
        assert L.omm_gpu_set_fp64_gemm(1, 16 * 384 * 256) == 0  # one 256-column panel at a time
        got, opa, opb, C0 = _run("t", "n", M, N, K, beta=0.5, seed=77)
    finally:
        assert L.omm_gpu_set_fp64_gemm(1, 0) == 0
    ref, mag = _exact(opa, opb, C0, 1.0, 0.5)
    assert np.all(np.abs(got - ref.astype(np.float64)) <= TOL * mag + 1e-300)


@pytest.mark.parametrize("M,N,K", [(200, 300, 777), (257, 513, 4099), (1536, 768, 2000)])
def test_sm_pair_kernel_matches_one_cta_kernel(M, N, K):
    """The 256 x 256 SM-pair kernel (cta_group::2) and the one-CTA kernel form the same exact
    integer products, so the FP64 results agree bit for bit (ragged pair tiles included)."""
    f, L = _fn()
    try:
        assert L.omm_gpu_tc_set_pairs(0) == 0
        one, opa, opb, C0 = _run("t", "n", M, N, K, beta=0.5, seed=M + K)
    finally:
        assert L.omm_gpu_tc_set_pairs(1) == 0
    pair, _, _, _ = _run("t", "n", M, N, K, beta=0.5, seed=M + K)
    assert np.array_equal(one, pair)
    ref, mag = _exact(opa, opb, C0, 1.0, 0.5)
    assert np.all(np.abs(pair - ref.astype(np.float64)) <= TOL * mag + 1e-300)


def _mag(A, B):
    aa, ab = np.abs(A), np.abs(B)
    return aa.max(axis=1)[:, None] * ab.sum(axis=0)[None, :] + aa.sum(axis=1)[:, None] * ab.max(axis=0)[None, :]


@pytest.mark.parametrize("opA", ["n", "t", "c"])
@pytest.mark.parametrize("opB", ["n", "t", "c"])
def test_complex_as_four_real_products(opA, opB):
    """Complex FP64 products with real scalars (MatrixSwitch mm_multiply on complex matrices) run as
    four real products of the parts: each of Re C = Ar Br -/+ Ai Bi and Im C = Ar Bi + Ai Br is held
    to the real products' bound, against a long-double complex product."""
    M, N, K = 256, 300, 2000
    rng = np.random.default_rng(hash((opA, opB, "z")) % 1000)
    ash = (M, K) if opA == "n" else (K, M)
    bsh = (K, N) if opB == "n" else (N, K)
    A = rng.standard_normal(ash) + 1j * rng.standard_normal(ash) * np.exp(rng.uniform(-2, 2, ash))
    B = rng.standard_normal(bsh) * np.exp(rng.uniform(-2, 2, bsh)) + 1j * rng.standard_normal(bsh)
    C0 = rng.standard_normal((M, N)) + 1j * rng.standard_normal((M, N))
    Ag, Bg, Cg = G.Matrix.from_numpy(A), G.Matrix.from_numpy(B), G.Matrix.from_numpy(C0)
    G.mm_multiply(Ag, opA, Bg, opB, Cg, alpha=0.75 + 0j, beta=-0.5 + 0j)
    got = Cg.numpy()
    op = {"n": lambda X: X, "t": lambda X: X.T, "c": lambda X: X.conj().T}
    opa, opb = op[opA](A), op[opB](B)
    la, lb = opa.astype(np.clongdouble), opb.astype(np.clongdouble)
    ref = 0.75 * (la @ lb) - 0.5 * C0.astype(np.clongdouble)
    ar, ai, br, bi = opa.real, opa.imag, opb.real, opb.imag
    mag_re = 0.75 * (_mag(ar, br) + _mag(ai, bi)) + np.abs(ref.real.astype(np.float64))
    mag_im = 0.75 * (_mag(ar, bi) + _mag(ai, br)) + np.abs(ref.imag.astype(np.float64))
    err_re = np.abs(got.real - ref.real.astype(np.float64))
    err_im = np.abs(got.imag - ref.imag.astype(np.float64))
    assert np.all(err_re <= TOL * mag_re + 1e-300), float(np.max(err_re / (mag_re + 1e-300)))
    assert np.all(err_im <= TOL * mag_im + 1e-300), float(np.max(err_im / (mag_im + 1e-300)))
