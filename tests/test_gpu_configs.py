"""Full-size checks of the adjoint configuration (complex Hermitian dense, m = 4096, n = 512,
16 sparse Hermitian perturbations V_k with 2 % fill and N(0, 0.01) entries).

Bars: the converged FP64 energy within 1e-9 relative of the eigenvalue sum; dE/dtheta_k
from the hand-written adjoint kernel (omm_gpu_energy_adjoint, SDDMM over V_k's nonzeros with
C recomputed into the density on the fly) within 1e-6 relative of
  * Re sum conj(D_min) o V_k with the density the solver returns (libOMM's gradient), all k;
  * central finite differences (h = 1e-5) of the exact eigenvalue sums, k = 0..3.
The eigenvalue problems are solved on the GPU in FP64 (torch / cuSOLVER)."""
import numpy as np
import pytest

import ommgpu as G
from ommgpu import synth

pytestmark = pytest.mark.gpu


def _reduced(Ht, L):
    import torch

    A = torch.linalg.solve_triangular(L, Ht, upper=False)
    return torch.linalg.solve_triangular(L, A.mH, upper=False)  # L^-1 H L^-H


def _dense_torch(V, m):
    import torch

    Vd = torch.zeros(m, m, dtype=torch.complex128, device="cuda")
    cols = np.repeat(np.arange(m), np.diff(V.colptr))
    Vd[torch.from_numpy(V.rowind.astype(np.int64)).cuda(), torch.from_numpy(cols).cuda()] = torch.from_numpy(
        V.val.astype(np.complex128)).cuda()
    return Vd


def test_adjoint_config_full_size():
    import torch

    p = synth.workload("zdense_4096")
    m, n = p.m, p.n
    assert (m, n, len(p.V)) == (4096, 512, 16)
    Hg, Sg = G.Matrix.from_numpy(p.H), G.Matrix.from_numpy(p.S)
    Cg, Dg = G.Matrix.allocate(n, m, "gzden"), G.Matrix.allocate(m, m, "gzden")
    e, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, cg_tol=1e-14, dealloc=True, m_storage="gzden")
    assert rc == 0
    assert abs(e - p.e_exact) <= 1e-9 * abs(p.e_exact), (e, p.e_exact)

    grad = G.energy_adjoint(m, n, Sg, Cg, [G.Matrix.from_csc(v) for v in p.V])

    # libOMM's gradient: Re sum conj(D) o V_k with the returned density
    D = Dg.numpy()
    for k, V in enumerate(p.V):
        cols = np.repeat(np.arange(m), np.diff(V.colptr))
        g_d = float(np.real(np.sum(np.conj(D[V.rowind, cols]) * V.val)))
        assert abs(grad[k] - g_d) <= 1e-6 * max(1.0, abs(g_d)), (k, grad[k], g_d)

    # central differences of the exact eigenvalue sums
    Ht = torch.from_numpy(np.ascontiguousarray(p.H)).cuda()
    L = torch.linalg.cholesky(torch.from_numpy(np.ascontiguousarray(p.S)).cuda())
    h = 1e-5
    for k in range(4):
        Vd = _dense_torch(p.V[k], m)
        ep = torch.linalg.eigvalsh(_reduced(Ht + h * Vd, L))[:n].sum().item()
        em = torch.linalg.eigvalsh(_reduced(Ht - h * Vd, L))[:n].sum().item()
        fd = (ep - em) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-6 * max(1.0, abs(fd)), (k, grad[k], fd)
        del Vd
    torch.cuda.empty_cache()
