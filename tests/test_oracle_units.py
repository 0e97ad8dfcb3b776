"""Unit checks of the oracle's building blocks against independent numpy arithmetic."""
import numpy as np
import pytest

import oracle as O
from ommgpu import synth


def rand_csc(rng, m, n, fill, cplx=False):
    import scipy.sparse as sp

    A = sp.random(m, n, density=fill, random_state=np.random.RandomState(rng.integers(1 << 30)), format="csc")
    if cplx:
        A = A + 1j * sp.random(m, n, density=fill, random_state=np.random.RandomState(rng.integers(1 << 30)),
                               format="csc").multiply(A != 0)
    A.sort_indices()
    return O.CSC(m, n, A.indptr.astype(np.int32), A.indices.astype(np.int32), np.ascontiguousarray(A.data)), A


def opm(a, op):
    return a if op == "n" else (a.T if op == "t" else a.conj().T)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("opA", ["n", "t", "c"])
@pytest.mark.parametrize("opB", ["n", "t", "c"])
def test_dense_times_csc(cplx, opA, opB):
    rng = np.random.default_rng(3)
    M, N, K = 7, 9, 11
    dt = np.complex128 if cplx else np.float64
    Ad = rng.standard_normal((M, K) if opA == "n" else (K, M)).astype(dt)
    if cplx:
        Ad = Ad + 1j * rng.standard_normal(Ad.shape)
    Bc, Bs = rand_csc(rng, *((K, N) if opB == "n" else (N, K)), 0.3, cplx)
    C0 = rng.standard_normal((M, N)).astype(dt)
    C = np.asfortranarray(C0.copy())
    O.mm_multiply(np.asfortranarray(Ad), opA, Bc, opB, C, 0.7, 0.3)
    ref = 0.7 * opm(Ad, opA) @ opm(Bs.toarray().astype(dt), opB) + 0.3 * C0
    if not cplx:
        ref = 0.7 * opm(Ad, opA) @ opm(Bs.toarray(), "t" if opB == "c" else opB) + 0.3 * C0
    assert np.allclose(C, ref, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("opA", ["n", "t", "c"])
def test_csc_times_dense(cplx, opA):
    rng = np.random.default_rng(4)
    M, N, K = 8, 5, 10
    dt = np.complex128 if cplx else np.float64
    Ac, As = rand_csc(rng, *((M, K) if opA == "n" else (K, M)), 0.3, cplx)
    B = rng.standard_normal((K, N)).astype(dt)
    C = np.zeros((M, N), dtype=dt, order="F")
    O.mm_multiply(Ac, opA, np.asfortranarray(B), "n", C, 1.0, 0.0)
    a = As.toarray().astype(dt)
    ref = opm(a, opA if cplx else ("t" if opA == "c" else opA)) @ B
    assert np.allclose(C, ref, rtol=1e-13, atol=1e-13)


def test_psp_alpha_zero_rule():
    # pspMspm.F90:114-116: alpha == 0 -> C = beta*C, and C untouched when beta == 0
    rng = np.random.default_rng(5)
    Bc, _ = rand_csc(rng, 6, 6, 0.5)
    A = np.asfortranarray(rng.standard_normal((4, 6)))
    C = np.asfortranarray(rng.standard_normal((4, 6)))
    C0 = C.copy()
    O.mm_multiply(A, "n", Bc, "n", C, 0.0, 0.0, psp=True)
    assert np.array_equal(C, C0)
    O.mm_multiply(A, "n", Bc, "n", C, 0.0, 2.0, psp=True)
    assert np.allclose(C, 2 * C0)


def test_quartic_minimum():
    # quartic with a known minimum: f(x) = (x-0.3)^2 ((x+1)^2 + 1) has its global minimum at 0.3
    p = np.polynomial.polynomial.polymul(np.polynomial.polynomial.polypow([-0.3, 1.0], 2), [2.0, 2.0, 1.0])
    x, fail = O.solve_quartic(p)
    assert not fail and abs(x - 0.3) < 1e-10
    # quadratic branch (c4 ~ 0): x = -c1/(2 c2)
    x, fail = O.solve_quartic([1.0, -2.0, 4.0, 0.0, 0.0])
    assert not fail and abs(x - 0.25) < 1e-15
    # c4 < 0 with one real stationary point -> fail
    x, fail = O.solve_quartic([0.0, 1.0, 0.0, 0.0, -1.0])
    assert fail


def test_lcg_matches_generator():
    for n, m in [(30, 60), (5, 7), (128, 832)]:
        assert np.array_equal(O.lcg_init(n, m), synth.lcg_c0(n, m))
        assert np.array_equal(O.lcg_init(n, m, True), synth.lcg_c0(n, m, True))


def test_lcg_first_values():
    # x1 = (1103515245*123456 + 12345) mod 2^31 etc. written out by hand
    x = 123456
    xs = []
    for _ in range(4):
        x = (1103515245 * x + 12345) % (1 << 31)
        xs.append(x / float(1 << 31))
    el0 = 0.5 * xs[0] if xs[1] - 0.5 >= 0 else -0.5 * xs[0]
    el1 = 0.5 * xs[2] if xs[3] - 0.5 >= 0 else -0.5 * xs[2]
    C = O.lcg_init(2, 3)
    s = 1e-2 / np.sqrt(3.0)
    assert C[0, 0] == el0 * s and C[1, 0] == el1 * s


@pytest.mark.parametrize("cplx", [False, True])
def test_calc_coeff_formulas(cplx):
    rng = np.random.default_rng(6)
    n = 9

    def r():
        a = rng.standard_normal((n, n))
        if cplx:
            a = a + 1j * rng.standard_normal((n, n))
        return np.asfortranarray(a)

    HW, SW, HWd, SWd, HWdd, SWdd = (r() for _ in range(6))
    c = O.calc_coeff(HW, SW, HWd, SWd, HWdd, SWdd)
    tr = lambda a: np.trace(a).real  # noqa: E731
    mt = lambda a, b: np.sum(np.conj(a) * b).real  # noqa: E731
    ref = [2 * tr(HW) - mt(HW, SW),
           2 * (2 * tr(HWd) - mt(SW, HWd) - mt(HW, SWd)),
           2 * (tr(HWdd) - mt(SWd.conj().T, HWd) - mt(SWd, HWd)) - mt(HWdd, SW) - mt(HW, SWdd),
           -2 * (mt(HWdd, SWd) + mt(SWdd, HWd)),
           -mt(HWdd, SWdd)]
    assert np.allclose(c, ref, rtol=1e-12, atol=1e-12)


def test_calc_G_formula():
    rng = np.random.default_rng(7)
    n, m = 5, 8
    HW, SW = rng.standard_normal((n, n)), rng.standard_normal((n, n))
    HC, SC = rng.standard_normal((n, m)), rng.standard_normal((n, m))
    G = O.calc_G(HW, SW, HC, SC)
    assert np.allclose(G, 4 * HC - 2 * SW @ HC - 2 * HW @ SC, rtol=1e-13, atol=1e-13)


def test_omm_energy_matches_eigensum_dense():
    p = synth.dense(200, 40, seed=9)
    orc = O.OmmOracle()
    C = np.zeros((p.n, p.m), order="F")
    D = np.zeros((p.m, p.m), order="F")
    e, rc = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False)
    assert rc == 0
    assert abs(e - p.e_exact) / abs(p.e_exact) < 1e-8
    # D is the S-projected density: tr(D S) = n
    assert abs(np.sum(D * p.S) - p.n) < 1e-6


@pytest.mark.parametrize("cplx", [False, True])
def test_oracle_flavour4_pw_preconditioner_converges(cplx):
    """The restated flavour 4 (calc_PW_precon, omm_ops.F90:1225-1334) reaches the eigenvalue sum."""
    import scipy.sparse as sp

    from ommgpu import synth

    p = synth.dense(120, 16, seed=39, complex_=cplx)
    tdiag = np.random.default_rng(40).uniform(0.0, 6.0, p.m)
    Tc = synth.CSCMatrix.from_scipy(sp.csc_matrix(sp.diags(tdiag.astype(complex) if cplx else tdiag)))
    orc = O.OmmOracle(nthreads=2)
    dt = complex if cplx else float
    C = np.zeros((p.n, p.m), dtype=dt, order="F")
    D = np.zeros((p.m, p.m), dtype=dt, order="F")
    e, rc = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False,
                    T=O.CSC(Tc.dim1, Tc.dim2, Tc.colptr, Tc.rowind, Tc.val.copy()), scale_T=3.0, flavour=4,
                    dealloc=True)
    assert rc == 0
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)
    with pytest.raises(RuntimeError):  # T dense: dcalc_PW_precon: invalid implementation
        orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False,
                T=np.asfortranarray(np.diag(tdiag).astype(dt)), scale_T=3.0, flavour=4, dealloc=True)
