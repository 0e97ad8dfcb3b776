"""Build the libOMM example problems from the committed fixtures.

Mirrors how libOMM/examples/example_gamma.F90:140-186 and
example_kpoints.F90:178-230 fill H and S with m_set_element, including the
second SCF step's rebuild with a -0.001 diagonal shift.
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _load():
    z = np.load(os.path.join(HERE, "examples.npz"))
    return {k: z[k] for k in z.files}


def golden() -> dict:
    with open(os.path.join(HERE, "examples.json")) as f:
        return json.load(f)


def gamma_HS(step: int = 1):
    """Real H, S (60 x 60, Fortran order) of example_gamma for SCF step 1 or 2; returns (m, n, H, S)."""
    z = _load()
    m, n = int(z["m"]), int(z["n"])
    H = np.zeros((m, m), order="F")
    S = np.zeros((m, m), order="F")
    i, j = z["gamma_idx"][:, 0] - 1, z["gamma_idx"][:, 1] - 1
    H[i, j] = z["gamma_val"][:, 0]
    S[i, j] = z["gamma_val"][:, 1]
    if step == 2:
        H[np.arange(m), np.arange(m)] += -0.001
    return m, n, H, S


def kpoints_HS(k: int, step: int = 1):
    """Complex H, S of example_kpoints for k-point k (1 or 2) and SCF step 1 or 2."""
    z = _load()
    m, n = int(z["m"]), int(z["n"])
    H = np.zeros((m, m), dtype=np.complex128, order="F")
    S = np.zeros((m, m), dtype=np.complex128, order="F")
    if k == 1:
        i, j = z["gamma_idx"][:, 0] - 1, z["gamma_idx"][:, 1] - 1
        H[i, j] = z["gamma_val"][:, 0]
        S[i, j] = z["gamma_val"][:, 1]
    else:
        i, j = z["kpoints_idx"][:, 0] - 1, z["kpoints_idx"][:, 1] - 1
        v = z["kpoints_val"]
        H[i, j] = v[:, 0] + 1j * v[:, 1]
        S[i, j] = v[:, 2] + 1j * v[:, 3]
    if step == 2:
        H[np.arange(m), np.arange(m)] += -0.001
    return m, n, H, S
