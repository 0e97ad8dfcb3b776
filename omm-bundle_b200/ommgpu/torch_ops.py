"""torch.autograd bindings of the library's hand-written derivative kernels (test binding).

* ``KimFunctional.apply(C, H, S)`` -> Omega(C) = tr[(2I - S_W) H_W] for a real
  C (torch tensor n x m, float64, CUDA); backward returns dOmega/dC = G from
  ``omm_gpu_functional_grad`` (libOMM's calc_G, omm_ops.F90:17-39).
* ``OmmEnergy.apply(theta, problem)`` -> the converged omm() energy of
  H(theta) = H0 + sum_k theta_k V_k; backward returns dE/dtheta_k from
  ``omm_gpu_energy_adjoint`` (sampled dense-dense kernel over V_k's nonzeros).

Both call the C ABI; tensors are handed over without copies through
``msw_register_gden`` (column-major views of torch memory).
"""
from __future__ import annotations

import numpy as np
import torch

import ommgpu as G
from ommgpu import synth


def _colmajor(t: torch.Tensor) -> torch.Tensor:
    """A contiguous (cols, rows) tensor whose memory is t (rows x cols) in column-major order."""
    return t.detach().t().contiguous()


class KimFunctional(torch.autograd.Function):
    @staticmethod
    def forward(ctx, C, H, S):
        if C.is_complex() or C.dtype != torch.float64 or not C.is_cuda:
            raise TypeError("KimFunctional expects a real float64 CUDA tensor C (n x m)")
        n, m = C.shape
        Cf = _colmajor(C)
        Gf = torch.empty((m, n), dtype=C.dtype, device=C.device)
        torch.cuda.synchronize()
        Cm = G.Matrix.register_gden(Cf.data_ptr(), n, m, False, keep=Cf)
        Gm = G.Matrix.register_gden(Gf.data_ptr(), n, m, False, keep=Gf)
        omega = G.functional_grad(m, n, H, S, Cm, Gm)
        ctx.save_for_backward(Gf)
        return C.new_tensor(omega)

    @staticmethod
    def backward(ctx, grad_out):
        (Gf,) = ctx.saved_tensors
        return grad_out * Gf.t(), None, None


def assemble(H0, V, theta):
    """H0 + sum_k theta_k V_k (CSCMatrix / ndarray inputs) as a device matrix handle."""
    th = [float(t) for t in theta]
    if isinstance(H0, synth.CSCMatrix):
        A = H0.to_scipy()
        for t, v in zip(th, V):
            if t != 0.0:
                A = A + t * v.to_scipy()
        return G.Matrix.from_csc(synth.CSCMatrix.from_scipy(A))
    A = np.array(H0, copy=True, order="F")
    for t, v in zip(th, V):
        if t != 0.0:
            A += t * v.to_dense()
    return G.Matrix.from_numpy(A)


class OmmEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, theta, problem: dict):
        H = assemble(problem["H0"], problem["V"], theta.detach().cpu().numpy())
        S = problem["S_handle"]
        m, n = problem["m"], problem["n"]
        lab = "gdden" if problem.get("real", True) else "gzden"
        Cm, Dm = G.Matrix.allocate(n, m, lab), G.Matrix.allocate(m, m, lab)
        e, rc = G.omm(m, n, H, S, True, Dm, False, 0.0, Cm, False, cg_tol=problem.get("cg_tol", 1e-14),
                      dealloc=True, m_operation=problem.get("label", "gpu"), m_storage=lab)
        Vh = problem.get("V_handles") or [G.Matrix.from_csc(v) for v in problem["V"]]
        problem["V_handles"] = Vh
        grad = G.energy_adjoint(m, n, S, Cm, Vh)
        ctx.save_for_backward(torch.as_tensor(grad, dtype=torch.float64, device=theta.device))
        return theta.new_tensor(e)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None
