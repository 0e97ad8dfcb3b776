"""Compute mu and the exact FP64 band energy of the lattice workloads and cache them.

``python make_spectra.py lattice_8x8x8 lattice_16x8x8 [--out file.json]`` runs one dense FP64
generalized eigensolve per workload (torch/cuSOLVER on a GPU when one is
present, else SciPy's dsygvd) and merges
{"mu", "e_exact", "gap", "spectrum", "n", "m"} into spectra.json, keyed by
workload name and seed.  synth.lattice() reads the cache so that the shift
mu = (lam_n + lam_{n+1})/2 does not need a dense eigensolve at every run.
"""
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from ommgpu import synth  # noqa: E402


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
    main(args, out=out)
