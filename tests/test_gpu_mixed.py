"""The mixed-precision solver ("gmx"): BF16 and split-BF16 stages on the tcgen05 GEMM and the
FP32 SpMM, finished in FP64.  It must reach the same converged energy as the FP64 path and the
oracle within 1e-9 relative (the bar for the mixed solver), with the density matrix
agreeing to the convergence level."""
import numpy as np
import pytest

import oracle as O
import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu


def solve(p, label, flavour=0, use_S=True, H=None, S=None):
    H = H if H is not None else p.H
    S = S if S is not None else p.S
    if isinstance(H, synth.CSCMatrix):
        Hg = G.Matrix.from_csc(H)
        Sg = G.Matrix.from_csc(S) if use_S else None
    else:
        Hg = G.Matrix.from_numpy(H)
        Sg = G.Matrix.from_numpy(S) if use_S else None
    lab = "gdden" if p.is_real else "gzden"
    Cg, Dg = G.Matrix.allocate(p.n, p.m, lab), G.Matrix.allocate(p.m, p.m, lab)
    e, rc = G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, flavour=flavour, dealloc=True,
                  m_operation=label, m_storage=lab)
    return e, rc, G.stats(), Dg.numpy()


@pytest.mark.parametrize("L", [(5, 5, 5), (6, 5, 5)])
def test_mixed_sparse_lattice_matches_fp64(L):
    p = synth.lattice(L, seed=101)
    e64, rc64, st64, D64 = solve(p, "gpu")
    emx, rcmx, stmx, Dmx = solve(p, "gmx")
    assert rc64 == 0 and rcmx == 0
    assert stmx["icg_low"] > 0 and stmx["icg_fp64"] >= 1
    assert abs(emx - e64) <= 1e-9 * abs(e64), (emx, e64, stmx)
    assert abs(emx - p.e_exact) <= 2e-9 * abs(p.e_exact)
    assert np.max(np.abs(Dmx - D64)) <= 1e-4 * np.max(np.abs(D64))


def test_mixed_dense_832_matches_oracle():
    p = synth.workload("dense_832")
    emx, rc, st, Dmx = solve(p, "gmx")
    orc = O.OmmOracle(nthreads=4)
    C = np.zeros((p.n, p.m), order="F")
    D = np.zeros((p.m, p.m), order="F")
    er, _ = orc.omm(p.m, p.n, p.H.copy(order="F"), p.S.copy(order="F"), True, D, False, 0.0, C, False, dealloc=True)
    assert rc == 0 and st["icg_low"] > 0
    assert abs(emx - er) <= 1e-9 * abs(er)
    assert abs(emx - p.e_exact) <= 2e-9 * abs(p.e_exact)


def test_mixed_hermitian_tile_skip():
    """n = 384 (a multiple of 128): the bf16 GEMM of [HWdd; SWdd] skips the tiles wholly below each
    half's diagonal (rows 256..383 against columns 0..255) and mirrors the lower triangles; the
    mixed energy matches the FP64 solve and the constructed eigenvalue sum."""
    p = synth.dense(2048, 384, seed=127)
    e64, rc64, _, D64 = solve(p, "gpu")
    emx, rc, st, Dmx = solve(p, "gmx")
    assert rc64 == 0 and rc == 0 and st["icg_low"] > 0
    assert abs(emx - e64) <= 1e-9 * abs(e64), (emx, e64, st)
    assert abs(emx - p.e_exact) <= 2e-9 * abs(p.e_exact)
    assert np.max(np.abs(Dmx - D64)) <= 1e-4 * np.max(np.abs(D64))


def test_mixed_cholesky_and_no_S():
    p = synth.dense(300, 40, seed=103)
    e64, _, _, _ = solve(p, "gpu", flavour=1, H=p.H.copy(order="F"), S=p.S.copy(order="F"))
    emx, rc, st, _ = solve(p, "gmx", flavour=1, H=p.H.copy(order="F"), S=p.S.copy(order="F"))
    assert rc == 0 and st["icg_low"] > 0
    assert abs(emx - e64) <= 1e-9 * abs(e64)
    w, V = np.linalg.eigh(p.S)
    Sih = (V / np.sqrt(w)) @ V.T
    Hp = np.asfortranarray(Sih @ p.H @ Sih)
    e64, _, _, _ = solve(p, "gpu", use_S=False, H=Hp)
    emx, rc, st, _ = solve(p, "gmx", use_S=False, H=Hp)
    assert rc == 0 and abs(emx - e64) <= 1e-9 * abs(e64)


def test_mixed_generic_sparse_pattern():
    """A CSC pattern without block structure (gather SpMM in the reduced stages)."""
    p = synth.dense(400, 50, seed=107)
    import scipy.sparse as sp

    Hs = sp.csc_matrix(np.where(np.abs(p.H) > 0.02, p.H, 0.0))
    Ss = sp.csc_matrix(np.where(np.abs(p.S) > 0.02, p.S, 0.0))
    Hc, Sc = synth.CSCMatrix.from_scipy(Hs), synth.CSCMatrix.from_scipy(Ss)
    try:
        np.linalg.cholesky(Sc.to_dense())
    except np.linalg.LinAlgError:
        pytest.skip("thresholded S is not positive definite")
    e64, rc64, _, _ = solve(p, "gpu", H=Hc, S=Sc)
    emx, rcmx, st, _ = solve(p, "gmx", H=Hc, S=Sc)
    assert rc64 == 0 and rcmx == 0
    assert abs(emx - e64) <= 1e-9 * abs(e64)


@pytest.mark.parametrize("variant", ["S", "no_S", "cholesky"])
def test_mixed_complex_dense_matches_fp64(variant):
    """Complex Hermitian problems run the reduced-precision stages as real GEMMs on
    [Re | Im] shadows (A') and [[Re | -Im]; [Im | Re]] shadows (B')."""
    p = synth.dense(360, 40, seed=109, complex_=True)
    kw = {}
    if variant == "no_S":
        kw = dict(use_S=False)
        w, V = np.linalg.eigh(p.H)
        exact = float(np.sort(w)[: p.n].sum())
    else:
        exact = p.e_exact
        if variant == "cholesky":
            kw = dict(flavour=1)
    H, S = p.H.copy(order="F"), p.S.copy(order="F")
    e64, rc64, st64, D64 = solve(p, "gpu", H=H.copy(order="F"), S=S.copy(order="F"), **kw)
    emx, rcmx, stmx, Dmx = solve(p, "gmx", H=H.copy(order="F"), S=S.copy(order="F"), **kw)
    assert rc64 == 0 and rcmx == 0
    assert stmx["icg_low"] > 0, stmx
    assert abs(emx - e64) <= 1e-9 * abs(e64), (emx, e64, stmx)
    assert abs(emx - exact) <= 2e-9 * abs(exact)
    assert np.max(np.abs(Dmx - D64)) <= 1e-4 * np.max(np.abs(D64))


def test_mixed_complex_adjoint_config():
    """The adjoint configuration (complex Hermitian dense, m = 4096, n = 512) under gmx: the
    FP64 energy of its C within 1e-9 of the FP64 path's."""
    p = synth.workload("zdense_4096")
    e64, rc64, st64, _ = solve(p, "gpu")
    emx, rcmx, stmx, _ = solve(p, "gmx")
    assert rc64 == 0 and rcmx == 0 and stmx["icg_low"] > 0
    assert abs(emx - e64) <= 1e-9 * abs(e64), (emx, e64, stmx)
    assert abs(emx - p.e_exact) <= 2e-9 * abs(p.e_exact)
