"""Generate the golden fixtures in tests/golden/ from the reference's own test files.

Run once where the reference tree is available, passing its root as
``--ref <path>``.  It reads, as data, the inputs and the asserted values of

* libOMM/examples/example_gamma.F90 + example_gamma.dat   (real, 60 x 60, n=30)
* libOMM/examples/example_kpoints.F90 + example_kpoints.dat (complex, 2 k-points)
* MatrixSwitch/examples/example_sdden.F90                  (dense API traces)

and writes

* ``examples.npz``  — the element lists of H and S exactly as the examples read
  them (example_gamma.F90:98-104, example_kpoints.F90:117-130);
* ``examples.json`` — the asserted constants and tolerances and the
  full-precision sample outputs printed in each example's header, each with the
  file:line it came from.

The GPU tests and bench never read the reference tree; they read these files.
"""
from __future__ import annotations

import argparse
import json
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_elements(path: str, ncols: int):
    # '(i2,1x,i2,1x,i4)' header then '(i2,1x,i2,k(1x,es10.3e2))' records
    with open(path) as f:
        lines = f.read().splitlines()
    m, n, ne = (int(x) for x in lines[0].split())
    idx = np.zeros((ne, 2), dtype=np.int32)
    val = np.zeros((ne, ncols), dtype=np.float64)
    for r, line in enumerate(lines[1 : 1 + ne]):
        idx[r, 0] = int(line[0:2])
        idx[r, 1] = int(line[3:5])
        for c in range(ncols):
            s = 6 + 11 * c
            val[r, c] = float(line[s : s + 10])
    return m, n, idx, val


def parse_param(src: str, name: str):
    # scalar 'name=v_dp' or array 'name(k)=(/v1_dp, &\n v2_dp/)' with continuation lines
    mt = re.search(r"::\s*%s(\(\d+\))?\s*=\s*(\(/.*?/\)|\S+)" % re.escape(name), src, re.S)
    if not mt:
        raise RuntimeError("parameter %s not found" % name)
    body = mt.group(2)
    nums = [float(x.replace("_dp", "")) for x in re.findall(r"-?\d+\.\d+(?:[dDeE][-+]?\d+)?_dp", body)]
    lineno = src[: mt.start()].count("\n") + 1
    return nums, lineno


def parse_samples(src: str):
    """Full-precision sample outputs from the '! Sample output:' header block."""
    out = []
    for lineno, line in enumerate(src.splitlines(), start=1):
        mt = re.match(r"!\s*(e_min|D_11|ED_11|res\d|E_11)\s*(\[[^\]]*\])?\s*:\s*(-?\d+\.\d+)(?:\s*,\s*(-?\d+\.\d+))?", line)
        if mt:
            out.append({"name": mt.group(1), "index": mt.group(2) or "", "re": float(mt.group(3)),
                        "im": float(mt.group(4)) if mt.group(4) else 0.0, "line": lineno})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="root of the reference source tree (omm-bundle checkout)")
    args = ap.parse_args()
    ex = os.path.join(args.ref, "libOMM", "examples")
    m, n, gidx, gval = read_elements(os.path.join(ex, "example_gamma.dat"), 2)
    m2, n2, kidx, kval = read_elements(os.path.join(ex, "example_kpoints.dat"), 4)
    assert (m, n) == (m2, n2)
    np.savez_compressed(os.path.join(HERE, "examples.npz"), m=m, n=n, gamma_idx=gidx, gamma_val=gval,
                        kpoints_idx=kidx, kpoints_val=kval)

    gsrc = open(os.path.join(ex, "example_gamma.F90")).read()
    ksrc = open(os.path.join(ex, "example_kpoints.F90")).read()
    ssrc = open(os.path.join(args.ref, "MatrixSwitch", "examples", "example_sdden.F90")).read()
    gold = {"source": "values asserted by the reference's example programs"}
    for tag, src, fname, names in (
        ("gamma", gsrc, "libOMM/examples/example_gamma.F90", ("e_min_check", "D_el_check", "ED_el_check")),
        ("kpoints", ksrc, "libOMM/examples/example_kpoints.F90", ("e_min_check", "D_el_check", "ED_el_check")),
        ("sdden", ssrc, "MatrixSwitch/examples/example_sdden.F90", ("res_check", "el_check")),
    ):
        entry = {}
        for nm in names:
            vals, ln = parse_param(src, nm)
            entry[nm] = {"values": vals, "cite": "%s:%d" % (fname, ln)}
        tol = re.search(r"tolerance\s*=\s*([0-9.]+)d([-+]?\d+)", src)
        entry["tolerance"] = float(tol.group(1)) * 10.0 ** int(tol.group(2))
        entry["tolerance_cite"] = "%s:%d" % (fname, src[: tol.start()].count("\n") + 1)
        entry["samples"] = parse_samples(src)
        entry["samples_cite"] = fname + " header 'Sample output'"
        gold[tag] = entry
    with open(os.path.join(HERE, "examples.json"), "w") as f:
        json.dump(gold, f, indent=1)
    print("wrote examples.npz and examples.json")


if __name__ == "__main__":
    main()
