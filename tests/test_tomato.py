"""tomato_TB (tomato/src/tomato_TB.F90:1-636): the GPU generator against the oracle's
restatement, on the synthetic templates of tests/golden/tomato (made by
tests/golden/make_tomato_templates.py; the reference ships no templates).

CPU tests: the oracle's own properties, and the host-only selection path of the library
(build_matrix false returns before any device work) against the oracle's scalars.
GPU tests: H and S element by element.  Bars: Gamma-point values bit-identical (the same
additions in the same order); k-point values within 4 ulp of the element's magnitude sum,
since the phases come from the device sincos instead of the host libm."""
import os

import numpy as np
import pytest

import ommgpu as G
import oracle as O

TPL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tomato")


def _args(**kw):
    a = dict(basedir=TPL, label="cube3d", switch1=False, frac_occ=0.0, num_orbs_per_atom=4, switch2=False,
             num_orbs=0, num_cells_dir=[2, 2, 2], switch3=False, sparsity=0.0, orb_r_cut=4.0, gamma_point=True,
             k_point=[0.0, 0.0, 0.0], defect=False, defect_perturbation=0.0)
    a.update(kw)
    return a


def _oracle(a, build=True):
    return O.tomato_TB(a["basedir"], a["label"], a["switch1"], a["frac_occ"], a["num_orbs_per_atom"], a["switch2"],
                       a["num_orbs"], a["num_cells_dir"], a["switch3"], a["sparsity"], a["orb_r_cut"],
                       a["gamma_point"], a["k_point"], a["defect"], a["defect_perturbation"], build_matrix=build)


def _gpu(a, storage, build=True):
    return G.tomato_TB(a["basedir"], a["label"], a["switch1"], a["frac_occ"], a["num_orbs_per_atom"], a["switch2"],
                       a["num_orbs"], a["num_cells_dir"], a["switch3"], a["sparsity"], a["orb_r_cut"],
                       a["gamma_point"], a["k_point"], a["defect"], a["defect_perturbation"], m_storage=storage,
                       build_matrix=build)


SCALARS = ("num_orbs_per_atom", "frac_occ", "num_orbs", "num_cells_dir", "orb_r_cut", "num_occ_states", "k_point")

SELECTIONS = [
    dict(),
    dict(switch1=True, frac_occ=0.9),  # 2/2 = 1.0 is closer than 2/4: the subset basis
    dict(switch1=True, frac_occ=0.75),  # halfway: the first size listed (4) wins ties
    dict(num_orbs_per_atom=3),  # |3-4| = |3-2|: the first closest, 4
    dict(switch2=True, num_orbs=8 * 27),  # 3 x 3 x 3 cells of 8 orbitals
    dict(switch2=True, num_orbs=200),
    dict(switch3=True, sparsity=0.0),  # the denser cutoff
    dict(switch3=True, sparsity=0.99),
    dict(orb_r_cut=3.3),  # nearest cutoff 2.5 (|330-250| < |330-400|)
    dict(label="chain1d", num_orbs_per_atom=3, num_cells_dir=[4, 4, 4], orb_r_cut=6.0, k_point=[0.3, 0.2, 0.1]),
    dict(label="chain1d", num_orbs_per_atom=3, switch2=True, num_orbs=31, orb_r_cut=3.0),
]


# ------------------------------------------------------------------------------ CPU
def test_oracle_gamma_symmetric_and_counts():
    """The templates list each element with its mirror, so H and S come out symmetric up to
    the order of the additions (several images of one element meet when a direction has one
    or two cells)."""
    r = _oracle(_args(num_cells_dir=[2, 3, 1]))
    H, S = r["H"], r["S"]
    assert r["num_orbs"] == 8 * 6 and H.shape == (48, 48)
    assert np.allclose(H, H.T, rtol=0, atol=1e-14) and np.allclose(S, S.T, rtol=0, atol=1e-14)
    assert r["num_occ_states"] == 2 * 2 * 6


def test_oracle_kpoint_hermitian_and_gamma_limit():
    a = _args(gamma_point=False, k_point=[0.25, 0.0, 0.5], num_cells_dir=[2, 2, 3])
    r = _oracle(a)
    assert np.allclose(r["H"], r["H"].conj().T, atol=1e-15)
    a0 = _args(gamma_point=False, k_point=[0.0, 0.0, 0.0], num_cells_dir=[2, 2, 3])
    g = _oracle(_args(num_cells_dir=[2, 2, 3]))
    assert np.array_equal(_oracle(a0)["H"].real, g["H"])


@pytest.mark.parametrize("sel", range(len(SELECTIONS)))
def test_selection_scalars_match_oracle(sel):
    """build_matrix false: the host-side selection of basis size, supercell and cutoff, and
    the element-count sparsity estimate, against the oracle (no device work)."""
    a = _args(**SELECTIONS[sel])
    ref = _oracle(a, build=False)
    got = _gpu(a, "sdden", build=False)
    for k in SCALARS + ("sparsity",):
        assert got[k] == ref[k], (k, got[k], ref[k])
    assert got["H"] is None and got["S"] is None


def test_missing_template_is_an_error():
    with pytest.raises(G.OmmError):
        _gpu(_args(label="nosuch"), "sdden", build=False)


# ------------------------------------------------------------------------------ GPU
def _dense(M):
    if M is None:
        return None
    lab = "gzden" if M.is_complex else "gdden"
    return M.copy(lab).numpy()


CASES = [
    ("gamma_full", dict(num_cells_dir=[2, 3, 2], orb_r_cut=4.0), "sdden"),
    ("gamma_cells1_wrap", dict(num_cells_dir=[1, 2, 1], orb_r_cut=4.0), "sdden"),
    ("gamma_subset_defect", dict(switch1=True, frac_occ=0.9, num_cells_dir=[3, 2, 2], defect=True,
                                 defect_perturbation=0.3), "pdcsc"),
    ("gamma_switch2_csc", dict(switch2=True, num_orbs=8 * 27, orb_r_cut=2.5), "sdcsc"),
    ("gamma_device_dense", dict(num_cells_dir=[2, 2, 2], defect=True, defect_perturbation=-1.5), "gdden"),
    ("kpoint_full", dict(gamma_point=False, k_point=[0.25, 0.1, 0.5], num_cells_dir=[2, 3, 2]), "szden"),
    ("kpoint_subset_defect", dict(gamma_point=False, k_point=[0.5, 0.5, 0.5], switch1=True, frac_occ=1.0,
                                  num_cells_dir=[2, 2, 3], defect=True, defect_perturbation=0.7), "pzcsc"),
    ("chain_nooverlap", dict(label="chain1d", num_orbs_per_atom=3, num_cells_dir=[1, 1, 7], orb_r_cut=6.0), "sdden"),
    ("chain_kpoint", dict(label="chain1d", num_orbs_per_atom=3, num_cells_dir=[5, 5, 3], orb_r_cut=6.0,
                          gamma_point=False, k_point=[0.3, 0.2, 0.1]), "gzden"),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,storage", CASES, ids=[c[0] for c in CASES])
def test_matrices_match_oracle(name, kw, storage):
    a = _args(**kw)
    ref = _oracle(a)
    got = _gpu(a, storage)
    for k in SCALARS + ("sparsity",):
        assert got[k] == ref[k], (k, got[k], ref[k])
    for M, R in ((got["H"], ref["H"]), (got["S"], ref["S"])):
        if R is None:
            assert M is None
            continue
        assert M.dims()[3] == storage.endswith("csc")
        D = _dense(M)
        assert D.shape == R.shape and np.iscomplexobj(D) == np.iscomplexobj(R)
        if a["gamma_point"]:
            assert np.array_equal(D, R), float(np.max(np.abs(D - R)))
        else:
            # the element's magnitude sum: |H| accumulated with |phase| = 1
            mag = np.abs(_oracle(dict(a, gamma_point=True))["H" if R is ref["H"] else "S"])
            mag = np.maximum(mag, np.abs(R))
            assert np.all(np.abs(D - R) <= 4 * np.finfo(float).eps * mag + 1e-300)
            assert np.array_equal(D == 0, R == 0)


@pytest.mark.gpu
def test_larger_supercell_symmetric():
    """8 x 8 x 8 cells of the 400 cutoff (4,096 orbitals): too slow for the pure-Python oracle.
    With at least three cells in each direction no two images of an element meet, so the
    template's mirror pairs make H and S exactly symmetric, and the row sums of S equal the
    template's per-orbital sums."""
    a = _args(num_cells_dir=[8, 8, 8], orb_r_cut=4.0)
    got = _gpu(a, "sdcsc")
    H, S = _dense(got["H"]), _dense(got["S"])
    assert H.shape == (4096, 4096)
    assert np.array_equal(H, H.T) and np.array_equal(S, S.T)
    num, ti, td, _ = O._tomato_elements(os.path.join(TPL, "cube3d_400_4.template"))
    per = np.zeros(8)
    for (o1, _o2, _d0, _d1, _d2), v in zip(ti, td):
        per[o1 - 1] += v[1]
    rows = S.sum(axis=1).reshape(512, 8)
    assert np.allclose(rows, per[None, :], rtol=0, atol=1e-12)
