"""Compute mu and the exact FP64 band energy of the lattice workloads and cache them.

``python make_spectra.py lattice_8x8x8 lattice_16x8x8 [--out file.json]`` runs one dense FP64
generalized eigensolve per workload (torch/cuSOLVER on a GPU when one is
present, else SciPy's dsygvd) and merges
{"mu", "e_exact", "gap", "spectrum", "n", "m"} into spectra.json, keyed by
workload name and seed.  synth.lattice() reads the cache so that the shift
mu = (lam_n + lam_{n+1})/2 does not need a dense eigensolve at every run.
``--certify-mu MU`` replaces the full eigensolve, for orders cuSOLVER's syevd rejects,
by an inertia count at MU and a Rayleigh-Ritz solve on the converged FP64 omm()
subspace (``certified`` below).
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from ommgpu import synth  # noqa: E402


def _inertia_below(Hd, Sd, mu):
    """Number of generalized eigenvalues of (H, S) below mu: the negative inertia of H - mu S
    (Sylvester's law with S positive definite), from a Bunch-Kaufman LDL^T on the GPU."""
    import numpy as np
    import torch

    A = Hd - mu * Sd
    LD, piv = torch.linalg.ldl_factor(A)
    del A
    d = LD.diagonal().cpu().numpy()
    e = LD.diagonal(-1).cpu().numpy()
    p = piv.cpu().numpy()
    del LD
    torch.cuda.empty_cache()
    neg, k, n = 0, 0, len(d)
    while k < n:
        if p[k] > 0:  # 1 x 1 block
            neg += d[k] < 0
            k += 1
        else:  # 2 x 2 block [[d_k, e_k], [e_k, d_k+1]]
            det = d[k] * d[k + 1] - e[k] * e[k]
            neg += 1 if det < 0 else (2 if d[k] < 0 else 0)
            k += 2
    return int(neg)


def certified(name, mu0, seed=synth.DEFAULT_SEED):
    """mu and the band energy where a dense eigensolve of the whole pencil is out of reach
    (cuSOLVER's syevd rejects m = 49,152): (1) the inertia of H - mu0 S shows exactly n
    eigenvalues below mu0, so mu0 lies in the gap; (2) the FP64 GPU omm() (flavour 0,
    cg_tol 1e-14) converges to the occupied subspace; (3) the Rayleigh-Ritz eigenvalues of
    (H - mu0 S, S) on that subspace (an n x n dense FP64 eigensolve) are the occupied
    eigenvalues to the subspace's accuracy, and their sum is the band energy."""
    import numpy as np
    import torch

    import ommgpu as G

    t = time.time()
    w = synth.WORKLOADS[name]
    prob = synth.lattice(w["L"], seed, name, compute_mu=False)
    n, m = prob.n, prob.m
    Hd = synth._dense_on_device(prob.H, "cuda")
    Sd = synth._dense_on_device(prob.S, "cuda")
    below = _inertia_below(Hd, Sd, mu0)
    del Hd, Sd
    torch.cuda.empty_cache()
    if below != n:
        raise RuntimeError("mu0 = %g has %d eigenvalues below it, not n = %d" % (mu0, below, n))
    H = synth.CSCMatrix(prob.H.dim1, prob.H.dim2, prob.H.colptr, prob.H.rowind, prob.H.val - mu0 * prob.S.val)
    Hg, Sg = G.Matrix.from_csc(H), G.Matrix.from_csc(prob.S)
    Cg, Dg = G.Matrix.allocate(n, m), G.Matrix.allocate(m, m)
    G.set_log(None)
    e_omm, rc = G.omm(m, n, Hg, Sg, True, Dg, False, 0.0, Cg, False, cg_tol=1e-14, dealloc=True)
    icg = G.stats()["icg"]
    HC, SC = G.Matrix.allocate(n, m), G.Matrix.allocate(n, m)
    G.psp_gemspm(n, m, m, Cg, "n", Hg, "n", HC, 1.0, 0.0)
    G.psp_gemspm(n, m, m, Cg, "n", Sg, "n", SC, 1.0, 0.0)
    C = torch.from_numpy(Cg.numpy()).cuda()
    HW = C @ torch.from_numpy(HC.numpy()).cuda().T
    SW = C @ torch.from_numpy(SC.numpy()).cuda().T
    HW = 0.5 * (HW + HW.T)
    SW = 0.5 * (SW + SW.T)
    L = torch.linalg.cholesky(SW)
    A = torch.linalg.solve_triangular(L, HW, upper=False)
    A = torch.linalg.solve_triangular(L, A.T, upper=False)
    ritz = torch.linalg.eigvalsh(0.5 * (A + A.T)).cpu().numpy()
    rec = {"mu": float(mu0), "e_exact": float(np.sum(ritz)), "gap": None,
           "spectrum": [None, float(ritz[-1] + mu0), None, None], "n": n, "m": m,
           "seconds": time.time() - t,
           "method": "inertia of H - mu S (LDL^T) = n; Rayleigh-Ritz on the FP64 omm subspace (cg_tol 1e-14)",
           "omm_energy": float(e_omm), "omm_status": int(rc), "omm_cg_steps": int(icg)}
    return rec


def main(names, seed=synth.DEFAULT_SEED, out=None):
    out = out or synth._SPECTRA
    for name in names:
        w = synth.WORKLOADS[name]
        t = time.time()
        prob = synth.lattice(w["L"], seed, name, compute_mu=False)
        import numpy as np

        ev = synth.generalized_eigvals(prob.H, prob.S)
        n = prob.n
        mu = 0.5 * (ev[n - 1] + ev[n])
        rec = {"mu": float(mu), "e_exact": float(np.sum(ev[:n] - mu)), "gap": float(ev[n] - ev[n - 1]),
               "spectrum": [float(ev[0]), float(ev[n - 1]), float(ev[n]), float(ev[-1])], "n": n, "m": prob.m,
               "seconds": time.time() - t}
        cache = {}
        if os.path.exists(out):
            with open(out) as f:
                cache = json.load(f)
        cache[synth.spectrum_key(name, seed)] = rec
        with open(out, "w") as f:
            json.dump(cache, f, indent=1, sort_keys=True)
        print(name, rec, flush=True)


if __name__ == "__main__":
    args = sys.argv[1:]
    out = None
    if "--out" in args:
        i = args.index("--out")
        out = args[i + 1]
        del args[i:i + 2]
    if "--certify-mu" in args:  # python make_spectra.py lattice_16x16x8 --certify-mu -0.347 [--out f]
        i = args.index("--certify-mu")
        mu0 = float(args[i + 1])
        del args[i:i + 2]
        out = out or synth._SPECTRA
        for name in args:
            rec = certified(name, mu0)
            cache = {}
            if os.path.exists(out):
                with open(out) as f:
                    cache = json.load(f)
            cache[synth.spectrum_key(name, synth.DEFAULT_SEED)] = rec
            with open(out, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
            print(name, rec, flush=True)
    else:
        main(args, out=out)
