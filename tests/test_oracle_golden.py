"""The CPU oracle reproduces the values the reference's own example programs assert.

* libOMM/examples/example_gamma.F90:51-53, :140-245 (flavours 0, 1, 3, two SCF
  steps and the energy-weighted density), tolerance 1e-4 (:269)
* libOMM/examples/example_kpoints.F90:66-70, :176-310 (complex, np=2)
* MatrixSwitch/examples/example_sdden.F90:41-44, :78-130 (traces of products, 1e-10)
"""
import numpy as np
import pytest

import oracle as O
from tests.golden.examples import gamma_HS, golden, kpoints_HS


def run_gamma_sequence(orc, flavour):
    """example_gamma.F90:134-245 for one flavour; returns [(e1, D11), (e2, D11)], ED11."""
    m, n, H, S = gamma_HS(1)
    C = np.zeros((n, m), order="F")
    D = np.zeros((m, m), order="F")
    ED = np.zeros((m, m), order="F")
    out = []
    for step in (1, 2):
        if step == 2:
            H[:] = gamma_HS(2)[2]
        e, rc = orc.omm(m, n, H, S, step == 1, D, False, 0.0, C, step == 2, flavour=flavour)
        assert rc == 0
        out.append((e, D[0, 0]))
    orc.omm(m, n, H, S, False, ED, True, 0.0, C, True, flavour=0, dealloc=True)
    return out, ED[0, 0]


@pytest.mark.parametrize("flavour", [0, 1, 3])
def test_gamma_example(flavour):
    g = golden()["gamma"]
    tol = g["tolerance"]
    res, ed = run_gamma_sequence(O.OmmOracle(), flavour)
    for i, (e, d) in enumerate(res):
        assert abs(e - g["e_min_check"]["values"][i]) <= tol
        assert abs(d - g["D_el_check"]["values"][i]) <= tol
    assert abs(ed - g["ED_el_check"]["values"][0]) <= tol


@pytest.mark.parametrize("flavour", [0, 1, 3])
def test_kpoints_example(flavour):
    g = golden()["kpoints"]
    tol = g["tolerance"]
    orc = O.OmmOracle()
    mats = {}
    for k in (1, 2):
        m, n, H, S = kpoints_HS(k, 1)
        mats[k] = dict(H=H, S=S, C=np.zeros((n, m), complex, order="F"), D=np.zeros((m, m), complex, order="F"),
                       ED=np.zeros((m, m), complex, order="F"))
    for i in (1, 2):
        for k in (1, 2):
            M = mats[k]
            if i == 2:
                M["H"][:] = kpoints_HS(k, 2)[2]
            e, rc = orc.omm(m, n, M["H"], M["S"], i == 1, M["D"], False, 0.0, M["C"], i == 2, flavour=flavour,
                            np_=2, ip=k)
            assert rc == 0
            idx = (k - 1) * 2 + (i - 1)
            assert abs(e - g["e_min_check"]["values"][idx]) <= tol
            assert abs(M["D"][0, 0].real - g["D_el_check"]["values"][idx]) <= tol
            assert abs(M["D"][0, 0].imag) <= tol
    for k in (1, 2):
        M = mats[k]
        orc.omm(m, n, M["H"], M["S"], False, M["ED"], True, 0.0, M["C"], True, flavour=0, np_=2, ip=k,
                dealloc=(k == 2))
        assert abs(M["ED"][0, 0].real - g["ED_el_check"]["values"][k - 1]) <= tol
        assert abs(M["ED"][0, 0].imag) <= tol


def sdden_inputs():
    """Deterministic inputs of example_sdden.F90:67-86 (rn = mod(4.2 rn, 1))."""
    N, M = 15, 8
    A = np.zeros((N, M), order="F")
    B = np.zeros((N, M), order="F")
    rn = 0.1
    for i in range(N):
        for j in range(M):
            rn = (4.2 * rn) % 1.0
            A[i, j] = rn
            rn = (4.2 * rn) % 1.0
            B[i, j] = rn
    return A, B


def test_sdden_example():
    g = golden()["sdden"]
    tol = g["tolerance"]
    A, B = sdden_inputs()
    res_check = g["res_check"]["values"][0]
    assert abs(O.mm_trace(A, B) - res_check) <= tol                      # res1
    D = np.zeros((8, 8), order="F")
    O.mm_multiply(A, "t", B, "n", D)                                      # res2
    assert abs(np.trace(D) - res_check) <= tol
    E = np.zeros((15, 15), order="F")
    O.mm_multiply(B, "n", A, "t", E)                                      # res3
    assert abs(np.trace(E) - res_check) <= tol
    assert abs(E[0, 0] - g["el_check"]["values"][0]) <= tol
