"""Generate tests/golden/purcell_gp.json from the reference's own Purcell data.

The reference ships the spectra of E at the dipole (fE.dat) and of the dipole
signal (fdip.dat), each `omega amplitude phase` after a three-line header, and
plots purcell.gp:3 from `paste fE.dat fdip.dat`:

    (($2*cos($3)*$5*sin($6)-$2*sin($3)*$5*cos($6))*$1/2/($5**2*$1**4/3)+1)

This script evaluates that expression column by column, exactly as written,
on every 100th row (omega > 0) and stores the inputs and results.  Run it
where the reference checkout is present:

    python tests/golden/make_purcell_fixture.py /path/to/DTmaxwell4
"""
import json
import math
import os
import sys


def rows(path):
    out = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            out.append([float(v) for v in line.split()])
    return out


def main(ref):
    fe, fd = rows(os.path.join(ref, "fE.dat")), rows(os.path.join(ref, "fdip.dat"))
    assert len(fe) == len(fd)
    data = []
    for q in range(1, len(fe), 100):
        c1, c2, c3 = fe[q]
        c4, c5, c6 = fd[q]
        assert c1 == c4 and c1 > 0
        val = (c2 * math.cos(c3) * c5 * math.sin(c6) - c2 * math.sin(c3) * c5 * math.cos(c6)) * c1 / 2 / (
            c5 ** 2 * c1 ** 4 / 3) + 1
        data.append([c1, c2, c3, c5, c6, val])
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "purcell_gp.json"), "w") as f:
        json.dump({"source": "fE.dat, fdip.dat, purcell.gp:3 of the reference",
                   "columns": ["omega", "amp_E", "phase_E", "amp_dip", "phase_dip", "purcell_gp"],
                   "rows": data}, f, indent=0)
    print(len(data), "rows")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_purcell_fixture.py <path of the DTmaxwell4 source tree>")
    main(sys.argv[1])
