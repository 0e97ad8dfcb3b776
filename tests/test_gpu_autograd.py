"""Derivatives through the torch.autograd test binding (GPU): dOmega/dC and dE/dtheta.

Bars: backward == libOMM's calc_G restated in the oracle (1e-11 relative); directional
and parameter gradients == central finite differences (h = 1e-5) within 1e-6 relative,
the finite differences taken both on the oracle's converged energies (libOMM restated)
and on the exact eigenvalue sums."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as O
import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu


def test_kim_functional_backward():
    import torch

    from ommgpu.torch_ops import KimFunctional

    p = synth.dense(140, 18, seed=71)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    rng = np.random.default_rng(72)
    C0 = rng.standard_normal((p.n, p.m)) * 0.05
    C = torch.tensor(C0, dtype=torch.float64, device="cuda", requires_grad=True)
    om = KimFunctional.apply(C, Hg, Sg)
    om.backward()
    HC, SC = C0 @ p.H, C0 @ p.S
    HW, SW = HC @ C0.T, SC @ C0.T
    ref = O.calc_G(HW, SW, HC, SC)
    g = C.grad.cpu().numpy()
    assert np.max(np.abs(g - ref)) <= 1e-11 * np.max(np.abs(ref))
    dC = rng.standard_normal(C0.shape)
    h = 1e-5

    def omega(X):
        hw, sw = X @ p.H @ X.T, X @ p.S @ X.T
        return 2 * np.trace(hw) - np.sum(hw * sw)

    fd = (omega(C0 + h * dC) - omega(C0 - h * dC)) / (2 * h)
    assert abs(fd - np.sum(g * dC)) <= 1e-6 * abs(fd)


@pytest.mark.parametrize("kind", ["dense", "lattice"])
def test_omm_energy_adjoint_vs_fd(kind):
    import torch

    from ommgpu.torch_ops import OmmEnergy

    if kind == "dense":
        p = synth.dense(150, 20, seed=81, nperturb=3)
        S_h = G.Matrix.from_numpy(p.S)
    else:
        p = synth.lattice((5, 5, 5), seed=82, norb=4, nocc=1, nperturb=3)
        S_h = G.Matrix.from_csc(p.S)
    prob = {"H0": p.H, "V": p.V, "S_handle": S_h, "m": p.m, "n": p.n, "cg_tol": 1e-14}
    theta = torch.zeros(len(p.V), dtype=torch.float64, device="cuda", requires_grad=True)
    E = OmmEnergy.apply(theta, prob)
    E.backward()
    g = theta.grad.cpu().numpy()
    Hd = p.H.to_dense() if isinstance(p.H, synth.CSCMatrix) else p.H
    Sd = p.S.to_dense() if isinstance(p.S, synth.CSCMatrix) else p.S
    h = 1e-5
    orc = O.OmmOracle(nthreads=4)
    for k, V in enumerate(p.V):
        Vd = V.to_dense()
        # exact: eigenvalue sums of the generalized problem
        ep = sl.eigh(Hd + h * Vd, Sd, eigvals_only=True)[: p.n].sum()
        em = sl.eigh(Hd - h * Vd, Sd, eigvals_only=True)[: p.n].sum()
        fd_exact = (ep - em) / (2 * h)
        assert abs(g[k] - fd_exact) <= 1e-6 * max(1.0, abs(fd_exact)), (k, g[k], fd_exact)
        # the restated libOMM's converged energies
        es = []
        for sgn in (1, -1):
            C = np.zeros((p.n, p.m), order="F")
            D = np.zeros((p.m, p.m), order="F")
            e, _ = orc.omm(p.m, p.n, np.asfortranarray(Hd + sgn * h * Vd), np.asfortranarray(Sd), True, D, False,
                           0.0, C, False, cg_tol=1e-14, dealloc=True)
            es.append(e)
        fd_omm = (es[0] - es[1]) / (2 * h)
        assert abs(g[k] - fd_omm) <= 1e-6 * max(1.0, abs(fd_omm)), (k, g[k], fd_omm)


def test_complex_energy_adjoint_vs_eigensum():
    p = synth.dense(96, 12, seed=91, complex_=True, nperturb=2)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Cg, Dg = G.Matrix.allocate(p.n, p.m, "gzden"), G.Matrix.allocate(p.m, p.m, "gzden")
    G.omm(p.m, p.n, Hg, Sg, True, Dg, False, 0.0, Cg, False, cg_tol=1e-14, dealloc=True)
    grad = G.energy_adjoint(p.m, p.n, Sg, Cg, [G.Matrix.from_csc(v) for v in p.V])
    h = 1e-5
    for k, V in enumerate(p.V):
        Vd = V.to_dense()
        ep = sl.eigh(p.H + h * Vd, p.S, eigvals_only=True)[: p.n].sum()
        em = sl.eigh(p.H - h * Vd, p.S, eigvals_only=True)[: p.n].sum()
        fd = (ep - em) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("n,cplx", [(3072, True), (6144, False)])
def test_energy_adjoint_column_of_48_kib(n, cplx):
    """The adjoint kernel keeps one density column (n values) in shared memory; n = 3072 complex
    and 6144 real make it exactly 48 KiB, past the default limit once static shared memory is
    added.  Checked against Re sum conj(D) o V with D = C^H (2I - C S C^H) C in torch FP64."""
    import torch

    m = n + 64
    rng = np.random.default_rng(n)
    dt = np.complex128 if cplx else np.float64
    C = rng.standard_normal((n, m)) + (1j * rng.standard_normal((n, m)) if cplx else 0)
    C = np.asfortranarray((C / np.sqrt(m)).astype(dt))
    V = synth.sparse_perturbations(m, 2, fill=4.0 / m, seed=7, complex_=cplx)
    Cg = G.Matrix.from_numpy(C)
    grad = G.energy_adjoint(m, n, None, Cg, [G.Matrix.from_csc(v) for v in V])
    Ct = torch.from_numpy(C).cuda()
    SW = Ct @ Ct.conj().T
    D = Ct.conj().T @ ((2.0 * torch.eye(n, dtype=Ct.dtype, device="cuda") - SW) @ Ct)
    for k, v in enumerate(V):
        rows, cols, vals = synth.csc_device_index(v, "cuda")
        ref = float(torch.real(torch.sum(torch.conj(D[rows, cols]) * vals)).item())
        assert abs(grad[k] - ref) <= 1e-10 * max(1.0, abs(ref)), (k, grad[k], ref)
