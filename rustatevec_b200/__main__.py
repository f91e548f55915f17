"""Command-line smoke run on the B200 engine, the counterpart of qsv's CLI
(crates/qsv-cli/src/main.rs:1-31): GHZ(n) (H on qubit 0, then CX(0, q) for q = 1..n-1; n from the
first argument, 4 when it is missing or not a number) in complex128, then its non-negligible
outcome probabilities and the norm, printed in the same format.

    python -m rustatevec_b200 [n]
"""
from __future__ import annotations

import sys

import numpy as np

from .backend import B200Backend
from .circuit import Circuit


def main(argv=None) -> int:
    args = sys.argv[1:] if argv is None else list(argv)
    try:
        n = int(args[0])
    except (IndexError, ValueError):
        n = 4
    c = Circuit(n)
    c.h(0)
    for q in range(1, n):
        c.cx(0, q)
    be = B200Backend(0, precision="f64")
    try:
        st = be.execute(c)
        p = be.probabilities(st)
        print(f"GHZ({n}) — non-negligible outcome probabilities:")
        for i in np.flatnonzero(p > 1e-12):
            print(f"  |{int(i):0{n}b}⟩ : {p[i]:.6f}")
        print(f"⟨ψ|ψ⟩ = {be.norm_sqr(st):.6f}")
        st.free()
    finally:
        be.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
