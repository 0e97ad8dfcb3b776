"""GPU parity tests: every entry point through the C ABI against the CPU oracle.

Bars: FP64 products and traces within 1e-12 relative of the oracle; omm()
energies within 1e-10 relative of the oracle on the same seeded inputs and
within the reference examples' 1e-4 of their asserted values.
"""
import numpy as np
import pytest

import oracle as O
import ommgpu as G
from ommgpu import synth
from tests.golden.examples import gamma_HS, golden, kpoints_HS

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def rand_csc(rng, m, n, fill, cplx=False):
    import scipy.sparse as sp

    A = sp.random(m, n, density=fill, random_state=np.random.RandomState(rng.integers(1 << 30)), format="csc")
    if cplx:
        A = A + 1j * A.multiply(rng.standard_normal(A.shape) > 0)
    A = sp.csc_matrix(A)
    A.sort_indices()
    return synth.CSCMatrix.from_scipy(A)


def rnd(rng, shape, cplx):
    a = rng.standard_normal(shape)
    if cplx:
        a = a + 1j * rng.standard_normal(shape)
    return np.asfortranarray(a)


def close(a, b, rtol=RTOL):
    scale = max(1.0, float(np.max(np.abs(b))))
    return float(np.max(np.abs(a - b))) <= rtol * scale


# ------------------------------------------------------------------ pspBLAS
@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("opA", ["n", "t", "c"])
@pytest.mark.parametrize("opB", ["n", "t", "c"])
def test_psp_gemspm_all_ops(cplx, opA, opB):
    rng = np.random.default_rng(11)
    M, N, K = 37, 53, 61
    A = rnd(rng, (M, K) if opA == "n" else (K, M), cplx)
    B = rand_csc(rng, *((K, N) if opB == "n" else (N, K)), 0.15, cplx)
    C0 = rnd(rng, (M, N), cplx)
    al, be = (0.7 - 0.2j, 0.3 + 0.1j) if cplx else (0.7, 0.3)
    ref = C0.copy(order="F")
    O.mm_multiply(A, opA, O.CSC(B.dim1, B.dim2, B.colptr, B.rowind, B.val), opB, ref, al, be, psp=True)
    Cg = G.Matrix.from_numpy(C0)
    G.psp_gemspm(M, N, K, G.Matrix.from_numpy(A), opA, G.Matrix.from_csc(B), opB, Cg, al, be)
    assert close(Cg.numpy(), ref)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("opA", ["n", "t", "c"])
@pytest.mark.parametrize("opB", ["n", "t"])
def test_psp_gespmm_all_ops(cplx, opA, opB):
    rng = np.random.default_rng(12)
    M, N, K = 41, 29, 47
    A = rand_csc(rng, *((M, K) if opA == "n" else (K, M)), 0.2, cplx)
    B = rnd(rng, (K, N) if opB == "n" else (N, K), cplx)
    C0 = rnd(rng, (M, N), cplx)
    ref = C0.copy(order="F")
    O.mm_multiply(O.CSC(A.dim1, A.dim2, A.colptr, A.rowind, A.val), opA, B, opB, ref, 1.5, -0.5, psp=True)
    Cg = G.Matrix.from_numpy(C0)
    G.psp_gespmm(M, N, K, G.Matrix.from_csc(A), opA, G.Matrix.from_numpy(B), opB, Cg, 1.5, -0.5)
    assert close(Cg.numpy(), ref)


def test_psp_alpha_zero_leaves_C():
    rng = np.random.default_rng(13)
    B = rand_csc(rng, 20, 20, 0.2)
    C0 = rnd(rng, (10, 20), False)
    Cg = G.Matrix.from_numpy(C0)
    G.psp_gemspm(10, 20, 20, G.Matrix.from_numpy(rnd(rng, (10, 20), False)), "n", G.Matrix.from_csc(B), "n", Cg,
                 0.0, 0.0)
    assert np.array_equal(Cg.numpy(), C0)


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("n", [1, 33, 200])
def test_block_sparse_spmm_column_groups(cplx, n):
    """Block-structured CSC (lattice H) uses the column-group kernel; compare with the oracle."""
    p = synth.lattice((5, 5, 5), seed=21, norb=24, nocc=1, compute_mu=False)
    Hc = p.H
    if cplx:
        Hc = synth.CSCMatrix(Hc.dim1, Hc.dim2, Hc.colptr, Hc.rowind, Hc.val * (1 + 0.5j))
    rng = np.random.default_rng(14)
    A = rnd(rng, (n, p.m), cplx)
    ref = np.zeros((n, p.m), dtype=A.dtype, order="F")
    O.mm_multiply(A, "n", O.CSC(Hc.dim1, Hc.dim2, Hc.colptr, Hc.rowind, Hc.val), "n", ref, 1.0, 0.0)
    Hg = G.Matrix.from_csc(Hc)
    Cg = G.Matrix.allocate(n, p.m, "gzden" if cplx else "gdden")
    G.mm_multiply(G.Matrix.from_numpy(A), "n", Hg, "n", Cg, 1.0, 0.0)
    assert close(Cg.numpy(), ref, 1e-12)


# ------------------------------------------------------------------ MatrixSwitch dense ops
@pytest.mark.parametrize("cplx", [False, True])
def test_dense_ops(cplx):
    rng = np.random.default_rng(15)
    A, B = rnd(rng, (30, 20), cplx), rnd(rng, (20, 30), cplx)
    C = rnd(rng, (30, 30), cplx)
    Ag, Bg, Cg = G.Matrix.from_numpy(A), G.Matrix.from_numpy(B), G.Matrix.from_numpy(C)
    G.mm_multiply(Ag, "n", Bg, "n", Cg, 2.0, 0.5)
    assert close(Cg.numpy(), 2 * A @ B + 0.5 * C)
    Dg = G.Matrix.from_numpy(rnd(rng, (20, 30), cplx))
    D0 = Dg.numpy()
    G.m_add(Ag, "c", Dg, 1.5, -1.0)
    assert close(Dg.numpy(), 1.5 * A.conj().T - D0)
    X = rnd(rng, (25, 25), cplx)
    Y = rnd(rng, (25, 25), cplx)
    Xg, Yg = G.Matrix.from_numpy(X), G.Matrix.from_numpy(Y)
    assert abs(G.m_trace(Xg) - np.trace(X)) < 1e-12 * 25
    assert abs(G.mm_trace(Xg, Yg) - np.sum(np.conj(X) * Y)) < 1e-11 * np.abs(X).sum()
    G.m_scale(Xg, 0.25)
    assert close(Xg.numpy(), 0.25 * X)
    G.m_set(Yg, "u", 3.0, 5.0)
    Yn = Yg.numpy()
    iu = np.triu_indices(25, 1)
    assert np.all(Yn[iu] == 3.0) and np.all(np.diag(Yn) == 5.0)
    assert np.array_equal(Yn[np.tril_indices(25, -1)], Y[np.tril_indices(25, -1)])
    G.m_set_element(Xg, 3, 4, 1.0, 2.0)
    assert abs(G.m_get_element(Xg, 3, 4) - (1.0 + 2.0 * 0.25 * X[2, 3])) < 1e-14


def test_host_storage_staging():
    """sdden matrices (host memory) are staged to the GPU and written back."""
    rng = np.random.default_rng(16)
    A, B = rnd(rng, (12, 9), False), rnd(rng, (9, 7), False)
    C = np.zeros((12, 7), order="F")
    G.mm_multiply(G.Matrix.register_sden(A), "n", G.Matrix.register_sden(B), "n", G.Matrix.register_sden(C), 1.0,
                  0.0, "lap")
    assert close(C, A @ B)


# ------------------------------------------------------------------ omm on the reference examples
def gpu_gamma_sequence(flavour, label="gpu"):
    m, n, H, S = gamma_HS(1)
    Hg, Sg = G.Matrix.from_numpy(H), G.Matrix.from_numpy(S)
    Cg = G.Matrix.allocate(n, m, "gdden")
    Dg = G.Matrix.allocate(m, m, "gdden")
    EDg = G.Matrix.allocate(m, m, "gdden")
    out = []
    for step in (1, 2):
        if step == 2:
            Hg = G.Matrix.from_numpy(gamma_HS(2)[2])
        e, rc = G.omm(m, n, Hg, Sg, step == 1, Dg, False, 0.0, Cg, step == 2, flavour=flavour, m_operation=label)
        assert rc == 0
        out.append((e, G.m_get_element(Dg, 1, 1), G.stats()["icg"], Dg.numpy(), Cg.numpy()))
    G.omm(m, n, Hg, Sg, False, EDg, True, 0.0, Cg, True, flavour=0, dealloc=True)
    return out, EDg.numpy()


def oracle_gamma_sequence(flavour):
    orc = O.OmmOracle()
    m, n, H, S = gamma_HS(1)
    C = np.zeros((n, m), order="F")
    D = np.zeros((m, m), order="F")
    ED = np.zeros((m, m), order="F")
    out = []
    for step in (1, 2):
        if step == 2:
            H = gamma_HS(2)[2]
        e, _ = orc.omm(m, n, H, S, step == 1, D, False, 0.0, C, step == 2, flavour=flavour)
        out.append((e, D[0, 0], orc.icg, D.copy(), C.copy()))
    orc.omm(m, n, H, S, False, ED, True, 0.0, C, True, flavour=0, dealloc=True)
    return out, ED


@pytest.mark.parametrize("flavour", [0, 1, 3])
def test_omm_gamma_example(flavour):
    g = golden()["gamma"]
    tol = g["tolerance"]
    gpu, ed = gpu_gamma_sequence(flavour)
    ref, ed_ref = oracle_gamma_sequence(flavour)
    for i in range(2):
        e, d11, icg, D, C = gpu[i]
        er, d11r, icgr, Dr, Cr = ref[i]
        assert abs(e - g["e_min_check"]["values"][i]) <= tol
        assert abs(d11 - g["D_el_check"]["values"][i]) <= tol
        assert abs(e - er) <= 1e-10 * abs(er)        # FP64 parity with the restated reference
        assert icg == icgr                            # same CG trajectory
        assert close(D, Dr, 1e-8) and close(C, Cr, 1e-8)
    assert abs(ed[0, 0] - g["ED_el_check"]["values"][0]) <= tol
    assert close(ed, ed_ref, 1e-8)


def test_omm_kpoints_example():
    g = golden()["kpoints"]
    tol = g["tolerance"]
    for flavour in (0, 1):
        H, S, C, D = {}, {}, {}, {}
        orc = O.OmmOracle()
        Ho, So, Co, Do = {}, {}, {}, {}
        for k in (1, 2):
            m, n, h, s = kpoints_HS(k, 1)
            H[k], S[k] = G.Matrix.from_numpy(h), G.Matrix.from_numpy(s)
            C[k] = G.Matrix.allocate(n, m, "gzden")
            D[k] = G.Matrix.allocate(m, m, "gzden")
            Ho[k], So[k] = h.copy(order="F"), s.copy(order="F")
            Co[k] = np.zeros((n, m), complex, order="F")
            Do[k] = np.zeros((m, m), complex, order="F")
        for i in (1, 2):
            for k in (1, 2):
                if i == 2:
                    h2 = kpoints_HS(k, 2)[2]
                    H[k] = G.Matrix.from_numpy(h2)
                    Ho[k] = h2.copy(order="F")
                e, rc = G.omm(m, n, H[k], S[k], i == 1, D[k], False, 0.0, C[k], i == 2, flavour=flavour, np_=2, ip=k)
                er, _ = orc.omm(m, n, Ho[k], So[k], i == 1, Do[k], False, 0.0, Co[k], i == 2, flavour=flavour,
                                np_=2, ip=k)
                idx = (k - 1) * 2 + (i - 1)
                assert rc == 0
                assert abs(e - g["e_min_check"]["values"][idx]) <= tol
                assert abs(e - er) <= 1e-10 * abs(er)
                d11 = G.m_get_element(D[k], 1, 1)
                assert abs(d11.real - g["D_el_check"]["values"][idx]) <= tol
        for k in (1, 2):
            ED = G.Matrix.allocate(m, m, "gzden")
            G.omm(m, n, H[k], S[k], False, ED, True, 0.0, C[k], True, flavour=0, np_=2, ip=k, dealloc=(k == 2))
            assert abs(G.m_get_element(ED, 1, 1).real - g["ED_el_check"]["values"][k - 1]) <= tol


def test_omm_host_storage_and_lcg():
    """sdden handles (the reference's own storage) go through the GPU with staging; the
    reference's LCG start (NORAND) makes the run reproduce the oracle's CG trajectory."""
    m, n, H, S = gamma_HS(1)
    C = np.zeros((n, m), order="F")
    D = np.zeros((m, m), order="F")
    e, rc = G.omm(m, n, G.Matrix.register_sden(H.copy(order="F")), G.Matrix.register_sden(S.copy(order="F")), True,
                  G.Matrix.register_sden(D), False, 0.0, G.Matrix.register_sden(C), False, m_storage="sdden",
                  m_operation="lap", dealloc=True)
    orc = O.OmmOracle()
    C2 = np.zeros((n, m), order="F")
    D2 = np.zeros((m, m), order="F")
    er, _ = orc.omm(m, n, H.copy(order="F"), S.copy(order="F"), True, D2, False, 0.0, C2, False, dealloc=True)
    assert rc == 0 and abs(e - er) <= 1e-10 * abs(er)
    assert close(C, C2, 1e-8) and close(D, D2, 1e-8)


# ------------------------------------------------------------------ omm on synthetic workloads
def test_omm_dense_832():
    p = synth.workload("dense_832")
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Cg, Dg = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True)
    orc = O.OmmOracle(nthreads=4)
    C = np.zeros((p.n, p.m), order="F")
    D = np.zeros((p.m, p.m), order="F")
    er, rcr = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False,
                      dealloc=True)
    assert rc == rcr == 0
    assert abs(e - er) <= 1e-10 * abs(er)
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)
    assert close(Dg.numpy(), D, 1e-7)


@pytest.mark.parametrize("cplx", [False, True])
def test_omm_dense_odd_n_staircase(cplx):
    """n = 257 splits into no equal blocks of 128 or more, so the Hermitian products ([HWdd; SWdd]
    and the W matrices) take the staircase of row blocks; energy and density against the oracle."""
    p = synth.dense(832, 257, seed=11, complex_=cplx)
    lab = "gzden" if cplx else "gdden"
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Cg, Dg = G.Matrix.allocate(p.n, p.m, lab), G.Matrix.allocate(p.m, p.m, lab)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True, m_storage=lab)
    orc = O.OmmOracle(nthreads=4)
    dt = np.complex128 if cplx else np.float64
    C = np.zeros((p.n, p.m), dtype=dt, order="F")
    D = np.zeros((p.m, p.m), dtype=dt, order="F")
    er, rcr = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False,
                      dealloc=True)
    assert rc == rcr == 0
    assert abs(e - er) <= 1e-10 * abs(er)
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)
    assert close(Dg.numpy(), D, 1e-7)


@pytest.mark.parametrize("cplx", [False, True])
def test_cholesky_flavour_blocked_reduction(cplx):
    """At m = 4,096 the Cholesky flavour reduces H block row by block row (the blocked sygst
    form); its energy matches the constructed eigenvalue sum and its density the basic
    flavour's."""
    p = synth.dense(4096, 128, seed=7, complex_=cplx)
    lab = "gzden" if cplx else "gdden"
    out = {}
    for flavour in (0, 1):
        Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
        Cg, Dg = G.Matrix.allocate(p.n, p.m, lab), G.Matrix.allocate(p.m, p.m, lab)
        e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, flavour=flavour, dealloc=True,
                      m_storage=lab)
        assert rc == 0
        out[flavour] = (e, Dg.numpy())
    e1, D1 = out[1]
    assert abs(e1 - p.e_exact) <= 1e-9 * abs(p.e_exact), (e1, p.e_exact)
    assert close(D1, out[0][1], 1e-4)


@pytest.mark.parametrize("cplx", [False, True])
def test_omm_sparse_lattice(cplx):
    """CSC H and S (the pdcsc path collapsed to one GPU) against the oracle's CSC loops."""
    p = synth.lattice((5, 5, 5), seed=31, norb=8, nocc=1)
    H, S = p.H, p.S
    if cplx:
        H = synth.CSCMatrix(H.dim1, H.dim2, H.colptr, H.rowind, H.val.astype(complex))
        S = synth.CSCMatrix(S.dim1, S.dim2, S.colptr, S.rowind, S.val.astype(complex))
    Hg, Sg = G.Matrix.from_csc(H), G.Matrix.from_csc(S)
    lab = "gzden" if cplx else "gdden"
    Cg, Dg = G.Matrix.allocate(p.n, p.m, lab), G.Matrix.allocate(p.m, p.m, lab)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True)
    icg = G.stats()["icg"]
    orc = O.OmmOracle(nthreads=4)
    dt = complex if cplx else float
    C = np.zeros((p.n, p.m), dtype=dt, order="F")
    D = np.zeros((p.m, p.m), dtype=dt, order="F")
    er, _ = orc.omm(p.m, p.n, O.CSC(H.dim1, H.dim2, H.colptr, H.rowind, H.val.copy()),
                    O.CSC(S.dim1, S.dim2, S.colptr, S.rowind, S.val.copy()), True, D, False, 0.0, C, False,
                    dealloc=True)
    assert rc == 0
    assert abs(e - er) <= 1e-10 * abs(er)
    assert icg == orc.icg
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)


@pytest.mark.parametrize("cplx", [False, True])
def test_density_blocked_large_m(cplx):
    """m >= 2048 takes the blocked density D = C^H (2I - SW) C (upper blocks + mirror; m = 2050
    leaves a ragged last block): D must equal the product rebuilt from the returned C."""
    m, n = 2050, 48
    p = synth.dense(m, n, seed=113, complex_=cplx)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    lab = "gzden" if cplx else "gdden"
    Cg, Dg = G.Matrix.allocate(n, m, lab), G.Matrix.allocate(m, m, lab)
    e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True, m_storage=lab)
    assert rc == 0
    C = Cg.numpy()
    SW = C @ p.S @ C.conj().T
    Dref = C.conj().T @ ((2.0 * np.eye(n) - SW) @ C)
    D = Dg.numpy()
    assert close(D, Dref, 1e-11)
    assert np.array_equal(np.tril(D, -1), np.triu(D, 1).conj().T)  # lower triangle mirrored exactly
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)


def test_omm_no_S_and_warm_start():
    """S absent (S = I) and a second call with init_C=False, new_S=False (warm start, omm.F90:363-367)."""
    p = synth.dense(160, 24, seed=41)
    w, V = np.linalg.eigh(p.S)
    # orthonormal problem: H' = S^-1/2 H S^-1/2, no S
    Sih = (V / np.sqrt(w)) @ V.T
    Hp = np.asfortranarray(Sih @ p.H @ Sih)
    Hg = G.Matrix.from_numpy(Hp)
    Cg, Dg = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    e1, _ = G.omm(p.m, p.n, Hg, None, True, Dg, False, 0.0, Cg, False)
    e2, _ = G.omm(p.m, p.n, Hg, None, False, Dg, False, 0.0, Cg, False, dealloc=True)
    orc = O.OmmOracle()
    C = np.zeros((p.n, p.m), order="F")
    D = np.zeros((p.m, p.m), order="F")
    r1, _ = orc.omm(p.m, p.n, Hp.copy(order="F"), None, True, D, False, 0.0, C, False)
    r2, _ = orc.omm(p.m, p.n, Hp.copy(order="F"), None, False, D, False, 0.0, C, False, dealloc=True)
    assert abs(e1 - r1) <= 1e-10 * abs(r1) and abs(e2 - r2) <= 1e-10 * abs(r2)


# ------------------------------------------------------------------ error behaviour
def test_errors_map_to_reference_die():
    m, n, H, S = gamma_HS(1)
    Hg, Sg = G.Matrix.from_numpy(H), G.Matrix.from_numpy(S)
    Cg, Dg = G.Matrix.allocate(n, m), G.Matrix.allocate(m, m)
    with pytest.raises(G.OmmError) as e:  # omm.F90:165
        G.omm(m, n, Hg, Sg, True, Dg, True, 0.0, Cg, False)
    assert e.value.code == -5
    with pytest.raises(G.OmmError) as e:  # omm.F90:148
        G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, flavour=7)
    assert e.value.code == -1
    Sbad = S.copy(order="F")
    Sbad[0, 0] = -5.0  # not positive definite -> dpotrf info != 0 (omm_ops.F90:302)
    with pytest.raises(G.OmmError) as e:
        G.omm(m, n, Hg, G.Matrix.from_numpy(Sbad), True, Dg, False, 0.0, Cg, False, flavour=1)
    assert e.value.code == -4
    G.finalize()
    # the library stays usable after errors
    e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True)
    assert rc == 0 and abs(e - golden()["gamma"]["e_min_check"]["values"][0]) < 1e-4


def test_line_search_failure_rescaling_matches_oracle():
    """A positive definite H and a large caller C make the quartic's leading coefficient negative
    with one real root: libOMM's ls_fail branch (omm.F90:472-480, 496-497, 511-512, 519-523)
    triples e_min and halves C.  The library takes it as often as the oracle (whose energy history
    shows each as a factor of 3) and ends at the same energy."""
    rng = np.random.default_rng(0)
    m, n = 60, 8
    A = rng.standard_normal((m, m))
    H = A @ A.T / m + 0.5 * np.eye(m)
    B = rng.standard_normal((m, m))
    S = np.eye(m) + 0.02 * (B + B.T)
    C0 = rng.standard_normal((n, m))
    orc = O.OmmOracle(nthreads=1)
    C = np.asfortranarray(C0.copy())
    D = np.zeros((m, m), order="F")
    er, rcr = orc.omm(m, n, H.copy(order="F"), S.copy(order="F"), True, D, False, 0.0, C, True, dealloc=True)
    h = np.array(orc.history)
    fails = sum(1 for i in range(1, len(h)) if h[i - 1] != 0 and abs(h[i] / h[i - 1] - 3.0) < 1e-9)
    # the history starts after the first step: a failure there triples the starting energy
    HW, SW = C0 @ H @ C0.T, C0 @ S @ C0.T
    e0 = 2.0 * np.trace(HW) - np.trace(HW @ SW)
    fails += int(abs(h[0] / (3.0 * e0) - 1.0) < 1e-9)
    assert rcr == 0 and fails >= 1
    Cg, Dg = G.Matrix.from_numpy(C0), G.Matrix.allocate(m, m)
    e, rc = G.omm(m, n, G.Matrix.from_numpy(H), G.Matrix.from_numpy(S), True, Dg, False, 0.0, Cg, True,
                  dealloc=True)
    st = G.stats()
    assert rc == 0
    assert st["ls_fail"] == fails, (st["ls_fail"], fails)
    assert abs(st["icg"] - orc.icg) <= 2, (st["icg"], orc.icg)
    assert abs(e - er) <= 1e-9, (e, er)


def test_nonfinite_input_returns_status():
    """A NaN in H makes the line-search coefficients non-finite: OMM_ERR_NONFINITE (-7) comes back
    (the reference would carry the NaN along), and the library solves the next problem."""
    m, n, H, S = gamma_HS(1)
    Hbad = H.copy(order="F")
    Hbad[3, 3] = np.nan
    Cg, Dg = G.Matrix.allocate(n, m), G.Matrix.allocate(m, m)
    with pytest.raises(G.OmmError) as e:
        G.omm(m, n, G.Matrix.from_numpy(Hbad), G.Matrix.from_numpy(S), True, Dg, False, 0.0, Cg, False,
              dealloc=True)
    assert e.value.code == -7
    Cg, Dg = G.Matrix.allocate(n, m), G.Matrix.allocate(m, m)
    e, rc = G.omm(m, n, G.Matrix.from_numpy(H), G.Matrix.from_numpy(S), True, Dg, False, 0.0, Cg, False,
                  dealloc=True)
    assert rc == 0 and abs(e - golden()["gamma"]["e_min_check"]["values"][0]) < 1e-4


# ------------------------------------------------------------------ derivatives
def test_functional_gradient_matches_calc_G_and_fd():
    p = synth.dense(120, 16, seed=51)
    rng = np.random.default_rng(52)
    C = np.asfortranarray(rng.standard_normal((p.n, p.m)) * 0.05)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Gg = G.Matrix.allocate(p.n, p.m)
    om = G.functional_grad(p.m, p.n, Hg, Sg, G.Matrix.from_numpy(C), Gg)
    Gn = Gg.numpy()
    HC, SC = C @ p.H, C @ p.S
    HW, SW = HC @ C.T, SC @ C.T
    assert abs(om - (2 * np.trace(HW) - np.sum(HW * SW))) < 1e-11 * abs(om)
    Gref = O.calc_G(HW, SW, HC, SC)
    assert close(Gn, Gref, 1e-11)
    # central finite difference along a random direction
    dC = np.asfortranarray(rng.standard_normal(C.shape))
    h = 1e-5

    def omega(Cx):
        hw = Cx @ p.H @ Cx.T
        sw = Cx @ p.S @ Cx.T
        return 2 * np.trace(hw) - np.sum(hw * sw)

    fd = (omega(C + h * dC) - omega(C - h * dC)) / (2 * h)
    assert abs(fd - np.sum(Gn * dC)) <= 1e-6 * abs(fd)


def test_energy_adjoint_matches_fd():
    p = synth.dense(150, 20, seed=61, nperturb=4)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Cg, Dg = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, cg_tol=1e-14, dealloc=True)
    Vg = [G.Matrix.from_csc(V) for V in p.V]
    grad = G.energy_adjoint(p.m, p.n, Sg, Cg, Vg)
    # exact reference: tr(D V) with D from the returned density matrix
    Dn = Dg.numpy()
    tr = np.array([np.sum(Dn * V.to_dense()) for V in p.V])
    assert np.allclose(grad, tr, rtol=1e-10, atol=1e-12)
    # central finite differences of the eigenvalue sum (h = 1e-5)
    import scipy.linalg as sl

    h = 1e-5
    for k, V in enumerate(p.V[:2]):
        Vd = V.to_dense()
        ep = sl.eigh(p.H + h * Vd, p.S, eigvals_only=True)[: p.n].sum()
        em = sl.eigh(p.H - h * Vd, p.S, eigvals_only=True)[: p.n].sum()
        fd = (ep - em) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * max(1.0, abs(fd))


# ------------------------------------------------------------------ omm_callback
@pytest.mark.parametrize("kind", ["lattice", "dense"])
def test_omm_callback_matches_omm(kind):
    """omm_callback with H(C, HC) = psp_gemspm / mm_multiply of the same H reproduces omm
    (same CG steps, same energy and density) and, through it, the oracle."""
    if kind == "lattice":
        p = synth.lattice((5, 5, 5), seed=33, norb=8, nocc=1)
        Hg, Sg = G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)

        def H(C, HC):
            G.psp_gemspm(p.n, p.m, p.m, C, "n", Hg, "n", HC, 1.0, 0.0)
    else:
        p = synth.dense(200, 30, seed=35)
        Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)

        def H(C, HC):
            G.mm_multiply(C, "n", Hg, "n", HC, 1.0, 0.0)
    calls = []

    def Hc(C, HC):
        calls.append(1)
        H(C, HC)

    C1, D1 = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    e1, rc1 = G.omm(p.m, p.n, Hg, Sg, True, D1, False, 0.0, C1, False, dealloc=True)
    icg1 = G.stats()["icg"]
    C2, D2 = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    e2, rc2 = G.omm_callback(p.m, p.n, Hc, Sg, True, D2, False, 0.0, C2, False, dealloc=True)
    assert rc1 == rc2 == 0
    assert G.stats()["icg"] == icg1
    assert icg1 <= len(calls) <= icg1 + 2  # HC, then HG of each search direction (omm.F90:353-457)
    assert abs(e1 - e2) <= 1e-13 * abs(e1)
    assert close(D2.numpy(), D1.numpy(), 1e-11)
    assert abs(e2 - p.e_exact) <= 1e-8 * abs(p.e_exact)


def test_omm_callback_flavours_and_errors():
    p = synth.dense(120, 16, seed=37)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)

    def H(C, HC):
        G.mm_multiply(C, "n", Hg, "n", HC, 1.0, 0.0)

    C, D = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    for fl in (1, 2, 4):  # omm_callback.F90:136-155: only 0 and 3
        with pytest.raises(G.OmmError) as ei:
            G.omm_callback(p.m, p.n, H, Sg, True, D, False, 0.0, C, False, flavour=fl, dealloc=True)
        assert ei.value.code == -1

    def bad(C, HC):
        raise ValueError("boom")

    with pytest.raises(G.OmmError) as ei:
        G.omm_callback(p.m, p.n, bad, Sg, True, D, False, 0.0, C, False, dealloc=True)
    assert ei.value.code == -8
    # the library stays usable, and flavour 3 (preconditioned) runs through the callback
    T = G.Matrix.from_numpy(np.eye(p.m))
    e, rc = G.omm_callback(p.m, p.n, H, Sg, True, D, False, 0.0, C, False, T=T, scale_T=10.0, flavour=3,
                           dealloc=True)
    e0, _ = G.omm(p.m, p.n, Hg, Sg, True, D, False, 0.0, C, False, T=T, scale_T=10.0, flavour=3, dealloc=True)
    assert rc == 0 and abs(e - e0) <= 1e-12 * abs(e0)


@pytest.mark.parametrize("cplx", [False, True])
def test_omm_flavour4_pw_preconditioner(cplx):
    """Flavour 4 (calc_PW_precon, omm_ops.F90:1225-1334: P on T's CSC pattern) against the oracle,
    with a diagonal kinetic-energy T (plane waves), dense H and S."""
    import scipy.sparse as sp

    p = synth.dense(180, 24, seed=39, complex_=cplx)
    rng = np.random.default_rng(40)
    tdiag = rng.uniform(0.0, 6.0, p.m)
    Tsp = sp.csc_matrix(sp.diags(tdiag.astype(complex) if cplx else tdiag))
    Tc = synth.CSCMatrix.from_scipy(Tsp)
    lab = "gzden" if cplx else "gdden"
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Tg = G.Matrix.from_csc(Tc)
    Cg, Dg = G.Matrix.allocate(p.n, p.m, lab), G.Matrix.allocate(p.m, p.m, lab)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, T=Tg, scale_T=3.0, flavour=4, dealloc=True,
                  m_storage=lab)
    icg = G.stats()["icg"]
    orc = O.OmmOracle(nthreads=4)
    dt = complex if cplx else float
    C = np.zeros((p.n, p.m), dtype=dt, order="F")
    D = np.zeros((p.m, p.m), dtype=dt, order="F")
    er, rcr = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False,
                      T=O.CSC(Tc.dim1, Tc.dim2, Tc.colptr, Tc.rowind, Tc.val.copy()), scale_T=3.0, flavour=4,
                      dealloc=True)
    assert rc == rcr == 0
    assert icg == orc.icg
    assert abs(e - er) <= 1e-10 * abs(er)
    assert close(Dg.numpy(), D, 1e-7)
    assert abs(e - p.e_exact) <= 1e-8 * abs(p.e_exact)
    # T must be CSC (dcalc_PW_precon: invalid implementation), and present
    with pytest.raises(G.OmmError):
        G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, T=G.Matrix.from_numpy(Tsp.toarray()),
              scale_T=3.0, flavour=4, dealloc=True, m_storage=lab)
    with pytest.raises(G.OmmError):
        G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, flavour=4, dealloc=True, m_storage=lab)


# ------------------------------------------------------------------ FP64 column-group kernel widths
@pytest.mark.parametrize("norb", [8, 16, 32])
def test_column_group_widths_single_product(norb):
    """Atom blocks of 8, 16 and 32 orbitals give column groups of G = 8, 16, 32 (each its own
    FP64 tensor-core kernel instance); psp_gemspm with alpha and beta against numpy."""
    p = synth.lattice((5, 5, 5), seed=23, norb=norb, nocc=1, compute_mu=False)
    Hg = G.Matrix.from_csc(p.H)
    info = G.spmm_plan_info(Hg)
    assert info["column_groups"] and info["G"] == norb and info["fill"] == 1.0, info
    rng = np.random.default_rng(norb)
    n = 150
    A = rnd(rng, (n, p.m), False)
    C0 = rnd(rng, (n, p.m), False)
    Cg = G.Matrix.from_numpy(C0)
    G.psp_gemspm(n, p.m, p.m, G.Matrix.from_numpy(A), "n", Hg, "n", Cg, 1.5, 0.5)
    ref = 1.5 * (A @ p.H.to_dense()) + 0.5 * C0
    assert close(Cg.numpy(), ref, 1e-12)


def test_plan_reuse_by_pattern_content():
    """Column groups are kept by pattern content: a second matrix with H's pattern and other
    values reuses them, and one of the same size whose pattern differs in a single row index
    gets its own; every product against numpy."""
    from ommgpu.synth import CSCMatrix

    p = synth.lattice((5, 5, 5), seed=41, norb=8, nocc=1, compute_mu=False)
    H = p.H
    rng = np.random.default_rng(41)
    n = 96
    A = rnd(rng, (n, p.m), False)
    Ag = G.Matrix.from_numpy(A)
    moved = H.rowind.copy()
    j = p.m // 2
    lo, hi = H.colptr[j], H.colptr[j + 1]
    free = np.setdiff1d(np.arange(p.m), H.rowind[lo:hi])
    moved[hi - 1] = free[-1]  # one entry of column j moves to a row it did not hold
    order = np.argsort(moved[lo:hi], kind="stable")
    moved[lo:hi] = moved[lo:hi][order]
    vals2 = H.val.copy()
    vals2[lo:hi] = vals2[lo:hi][order]
    cases = [CSCMatrix(H.dim1, H.dim2, H.colptr, H.rowind, H.val),
             CSCMatrix(H.dim1, H.dim2, H.colptr, H.rowind, 2.0 * H.val + 0.25),
             CSCMatrix(H.dim1, H.dim2, H.colptr, moved, vals2)]
    for B in cases:
        Bg = G.Matrix.from_csc(B)
        Cg = G.Matrix.allocate(n, p.m)
        G.psp_gemspm(n, p.m, p.m, Ag, "n", Bg, "n", Cg, 1.0, 0.0)
        assert close(Cg.numpy(), A @ B.to_dense(), 1e-12)


@pytest.mark.parametrize("norb", [16, 32])
def test_omm_sparse_lattice_group_widths(norb):
    """omm() on lattices whose H and S take the fused (H, S) FP64 kernel with G = 16, 32,
    against the oracle's CSC loops: energy within 1e-10, same CG steps."""
    p = synth.lattice((5, 5, 5), seed=35, norb=norb, nocc=1)
    Hg, Sg = G.Matrix.from_csc(p.H), G.Matrix.from_csc(p.S)
    assert G.spmm_plan_info(Hg)["G"] == norb
    Cg, Dg = G.Matrix.allocate(p.n, p.m), G.Matrix.allocate(p.m, p.m)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, dealloc=True)
    icg = G.stats()["icg"]
    orc = O.OmmOracle(nthreads=4)
    C = np.zeros((p.n, p.m), order="F")
    D = np.zeros((p.m, p.m), order="F")
    er, _ = orc.omm(p.m, p.n, O.CSC(p.H.dim1, p.H.dim2, p.H.colptr, p.H.rowind, p.H.val.copy()),
                    O.CSC(p.S.dim1, p.S.dim2, p.S.colptr, p.S.rowind, p.S.val.copy()), True, D, False, 0.0, C,
                    False, dealloc=True)
    assert rc == 0
    assert abs(e - er) <= 1e-10 * abs(er)
    assert icg == orc.icg
