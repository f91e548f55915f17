"""Writes the golden fixtures under tests/golden/.

known_answers.json — the known answers the reference's own tests assert, transcribed with the
file:line of the assertion (paths inside the qsv project). The reference (Rust) cannot be
compiled in this environment, so these pins are what anchors the oracle.

oracle_states.npz — final states of a few seeded circuits computed by the oracle's RefBackend
restatement in FP64: regression vectors for the oracle itself and for the GPU tests.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

R2 = 1.0 / math.sqrt(2.0)

KNOWN = {
    "bell": {
        "cite": "crates/qsv-core/tests/oracle.rs:12-25",
        "n": 2, "ops": [["h", [0]], ["cx", [0, 1]]], "tol": 1e-12,
        "amps": {"0": [R2, 0.0], "1": [0.0, 0.0], "2": [0.0, 0.0], "3": [R2, 0.0]}, "norm": 1.0,
    },
    "ghz3": {
        "cite": "crates/qsv-core/tests/oracle.rs:27-43",
        "n": 3, "ops": [["h", [0]], ["cx", [0, 1]], ["cx", [0, 2]]], "tol": 1e-12,
        "amps": {"0": [R2, 0.0], "7": [R2, 0.0], **{str(i): [0.0, 0.0] for i in range(1, 7)}},
    },
    "x_self_inverse": {
        "cite": "crates/qsv-core/tests/oracle.rs:45-53",
        "n": 4, "ops": [["x", [2]], ["x", [2]]], "tol": 1e-12, "amps": {"0": [1.0, 0.0]}, "norm": 1.0,
    },
    "cx_on_zero_is_noop": {
        "cite": "crates/qsv-core/tests/oracle.rs:55-62",
        "n": 2, "ops": [["cx", [0, 1]]], "tol": 1e-12, "amps": {"0": [1.0, 0.0]},
    },
    "rx_pi": {
        "cite": "crates/qsv-core/tests/oracle.rs:64-72",
        "n": 1, "ops": [["rx", [0], math.pi]], "tol": 1e-12, "amps": {"0": [0.0, 0.0], "1": [0.0, -1.0]},
    },
    "norm_mixed": {
        "cite": "crates/qsv-core/tests/oracle.rs:74-91",
        "n": 4, "ops": [["h", [0]], ["rx", [1], 0.4], ["ry", [2], 1.1], ["cx", [0, 1]], ["cz", [1, 2]],
                        ["rzz", [2, 3], 0.7], ["swap", [0, 3]], ["t", [2]]],
        "tol": 1e-10, "amps": {}, "norm": 1.0,
    },
    "ghz6": {
        "cite": "crates/qsv-core/tests/equivalence.rs:136-146",
        "n": 6, "ops": [["h", [0]]] + [["cx", [0, q]] for q in range(1, 6)], "tol": 1e-12,
        "amps": {"0": [R2, 0.0], "63": [R2, 0.0]}, "others_abs2_below": 1e-24,
    },
}

QFT_UNIFORM = {"cite": "crates/qsv-core/tests/equivalence.rs:108-120", "ns": [1, 2, 3, 5, 8], "tol": 1e-12}
EXPZ_GHZ5 = {"cite": "crates/qsv-core/tests/sampling.rs:49-58", "n": 5,
             "masks": [1, 3, 15, 31], "values": [0.0, 1.0, 1.0, 0.0], "tol": 1e-9}
EXPZ_BASIC = {"cite": "crates/qsv-core/src/sample.rs:260-270",
              "cases": [[[1.0, 0.0, 0.0, 0.0], 1, 1.0], [[1.0, 0.0, 0.0, 0.0], 3, 1.0],
                        [[0.5, 0.0, 0.0, 0.5], 1, 0.0], [[0.5, 0.0, 0.0, 0.5], 3, 1.0]], "tol": 1e-12}
CX_PERMUTATION = {"cite": "crates/qsv-core/src/gate.rs:193-205", "col_to_row": [0, 3, 2, 1]}
IS_DIAGONAL = {"cite": "crates/qsv-core/src/gate.rs:223-239",
               "diagonal": [["z", 0], ["s", 0], ["t", 0], ["rz", 0.3], ["phase", 1.1], ["cz", 0],
                            ["rzz", 0.5], ["cphase", 0.9]],
               "dense": [["h", 0], ["x", 0], ["rx", 0.4], ["cx", 0], ["swap", 0]]}
LAYOUT = {"cite": "crates/qsv-core/src/state/layout.rs:136-193",
          "insert_zero_bit": [[11, 2, 19]], "gather_bits": [[37, [0, 2, 5], 7]],
          "tiles": {"n": 4, "targets": [1, 3]}}
COMPLEX_MUL = {"cite": "crates/qsv-core/src/complex.rs:110-115", "a": [1.0, 2.0], "b": [3.0, 4.0], "ab": [-5.0, 10.0]}
FUSION_COUNTS = {"cite": "crates/qsv-core/src/fusion.rs:162-185",
                 "qft6_default_reduces": True, "disjoint_h_max1_count": 2}


def main():
    out = {"circuits": KNOWN, "qft_uniform": QFT_UNIFORM, "expz_ghz5": EXPZ_GHZ5, "expz_basic": EXPZ_BASIC,
           "cx_permutation": CX_PERMUTATION, "is_diagonal": IS_DIAGONAL, "layout": LAYOUT,
           "complex_mul": COMPLEX_MUL, "fusion_counts": FUSION_COUNTS}
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)

    import oracle
    from rustatevec_b200.circuits import random_circuit, qft
    arrays = {}
    specs = [(6, 40, 1), (8, 60, 2), (10, 80, 9000), (7, 50, 0xC0FFEE)]
    for n, depth, seed in specs:
        re, im = oracle.run(random_circuit(n, depth, seed), oracle.REF, oracle.F64)
        arrays[f"random_{n}_{depth}_{seed}"] = re + 1j * im
    re, im = oracle.run(qft(9), oracle.REF, oracle.F64)
    arrays["qft_9"] = re + 1j * im
    np.savez_compressed(os.path.join(HERE, "oracle_states.npz"), **arrays)
    print("wrote", sorted(arrays))


if __name__ == "__main__":
    main()
