"""Properties of the seeded synthetic workloads (no GPU)."""
import numpy as np
import pytest

from ommgpu import synth


def test_lattice_structure_small():
    p = synth.lattice((5, 5, 5), seed=2, norb=8, nocc=1)
    assert p.m == 125 * 8 and p.n == 125
    # 33 neighbour blocks of 8 rows in every column
    assert np.all(np.diff(p.H.colptr) == 33 * 8)
    Hd, Sd = p.H.to_dense(), p.S.to_dense()
    assert np.array_equal(Hd, Hd.T) and np.array_equal(Sd, Sd.T)
    w = np.linalg.eigvalsh(Sd)
    assert w.min() > 0.3
    # mu puts exactly n generalized eigenvalues below zero
    import scipy.linalg as sl

    ev = sl.eigh(Hd, Sd, eigvals_only=True)
    assert np.sum(ev < 0) == p.n
    assert abs(np.sum(ev[: p.n]) - p.e_exact) < 1e-9 * abs(p.e_exact)


def test_lattice_needs_side5():
    with pytest.raises(ValueError):
        synth.lattice((4, 5, 5), compute_mu=False)


def test_named_lattice_is_cached():
    for name in ("lattice_8x8x8", "lattice_16x8x8"):
        key = synth.spectrum_key(name, synth.DEFAULT_SEED)
        if key not in synth._load_spectra():
            pytest.skip("spectrum of %s not cached yet" % name)


def test_dense_constructed_spectrum():
    p = synth.dense(120, 20, seed=4)
    import scipy.linalg as sl

    ev = sl.eigh(p.H, p.S, eigvals_only=True)
    assert abs(np.sum(ev[: p.n]) - p.e_exact) < 1e-9 * abs(p.e_exact)
    assert np.sum(ev < 0) == p.n


def test_complex_dense_hermitian():
    p = synth.dense(64, 8, seed=5, complex_=True, nperturb=3)
    assert np.allclose(p.H, p.H.conj().T)
    for V in p.V:
        Vd = V.to_dense()
        assert np.allclose(Vd, Vd.conj().T)
