"""Writes the synthetic tight-binding templates under tests/golden/tomato/ that the tomato_TB
tests read.  The reference ships no template files, so these are made up: seeded random
elements in the reference's own file formats (tomato_TB.F90:124-180 for <label>_template.info,
:339-378 for <label>_<cutoff>_<size>.template, one record '(2x,i10)' num_template then
'(i3,4(1x,i3),2(1x,es10.3e2))' per element, the second value only when an overlap is present).

Systems:
  cube3d  3 periodic directions, 2 atoms per cell, 2 occupied states per atom, cutoffs
          250 / 400, basis sizes 4 (full) and 2 (a subset of the 4-orbital basis: orbitals 1, 3),
          with an overlap; the 250 file has nearest-cell images only, the 400 file every
          image in -1..1, some elements listed twice so contributions add.
  chain1d one periodic direction (the third, as tomato_TB.F90:233-245 orders them), 1 atom
          per cell, 1 occupied state, cutoffs 300 / 600, basis size 3, no overlap; images up
          to 2 cells away.

Run: python tests/golden/make_tomato_templates.py
"""
import itertools
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "tomato")


def _fmt_line(o1, o2, d, vals):
    s = "%3d %3d %3d %3d %3d" % (o1, o2, d[0], d[1], d[2])
    for v in vals:
        s += " %10.3E" % v
    return s


def _elements(rng, norb_cell, offsets, overlap, dup_every=0):
    """Hermitian-looking element lists: (o1, o2, d) and (o2, o1, -d) carry the same value."""
    seen, groups = set(), []
    for d in offsets:
        for o1 in range(1, norb_cell + 1):
            for o2 in range(1, norb_cell + 1):
                key = (o1, o2, d)
                if key in seen:
                    continue
                mirror = (o2, o1, tuple(-x for x in d))
                dist = sum(abs(x) for x in d)
                h = float(rng.normal(-1.0, 0.5)) / (1 + dist) if (o1 != o2 or dist) else float(rng.normal(0.0, 1.0))
                s = (1.0 if (o1 == o2 and dist == 0) else float(rng.normal(0.0, 0.05)) / (1 + dist))
                # the values are written with 4 significant digits: round here so the mirror is exact
                h, s = float("%10.3E" % h), float("%10.3E" % s)
                g = [(o1, o2, d, [h, s] if overlap else [h])]
                seen.add(key)
                if mirror not in seen:
                    g.append((mirror[0], mirror[1], mirror[2], [h, s] if overlap else [h]))
                    seen.add(mirror)
                groups.append(g)
    if dup_every:  # a few repeated records (with their mirrors): the generator adds every record
        groups += [groups[i] for i in range(0, len(groups), dup_every)]
    return [e for g in groups for e in g]


def _write(path, elems):
    with open(path, "w") as f:
        f.write("  %10d\n" % len(elems))
        for o1, o2, d, vals in elems:
            f.write(_fmt_line(o1, o2, d, vals) + "\n")


def main():
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(20261203)
    # cube3d
    with open(os.path.join(OUT, "cube3d_template.info"), "w") as f:
        f.write("3\n2\n2\n2\n250\n400\n2\n4\n2 4 1 3\n")
    near = [d for d in itertools.product((-1, 0, 1), repeat=3) if sum(abs(x) for x in d) <= 1]
    full = list(itertools.product((-1, 0, 1), repeat=3))
    _write(os.path.join(OUT, "cube3d_250_4.template"), _elements(rng, 8, near, True))
    _write(os.path.join(OUT, "cube3d_400_4.template"), _elements(rng, 8, full, True, dup_every=37))
    # chain1d
    with open(os.path.join(OUT, "chain1d_template.info"), "w") as f:
        f.write("1\n1\n1\n2\n300\n600\n1\n3\n")
    _write(os.path.join(OUT, "chain1d_300_3.template"), _elements(rng, 3, [(0, 0, -1), (0, 0, 0), (0, 0, 1)], False))
    _write(os.path.join(OUT, "chain1d_600_3.template"),
           _elements(rng, 3, [(0, 0, d) for d in range(-2, 3)], False))


if __name__ == "__main__":
    main()
