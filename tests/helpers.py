"""Shared test helpers: an independent numpy contraction (third oracle) and comparisons."""
from __future__ import annotations

import json
import os

import numpy as np

from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def known_answers() -> dict:
    with open(os.path.join(GOLDEN, "known_answers.json")) as f:
        return json.load(f)


def circuit_from_spec(n, ops) -> Circuit:
    c = Circuit(n)
    for op in ops:
        name, qs = op[0], op[1]
        g = G.LIBRARY[name](op[2]) if len(op) > 2 else G.LIBRARY[name]()
        c.push(g, qs)
    return c


def numpy_apply(psi: np.ndarray, n: int, mat: np.ndarray, qubits) -> np.ndarray:
    """Apply a gate by tensordot on the state reshaped to n axes of size 2 (axis n-1-q is qubit q)."""
    m = len(qubits)
    t = psi.reshape((2,) * n)
    u = mat.reshape((2,) * (2 * m))
    # gate index bit j <-> qubits[j]; in the reshaped matrix the row axes are ordered MSB first,
    # i.e. row axis a corresponds to bit (m-1-a) -> qubit qubits[m-1-a]
    col_axes = list(range(m, 2 * m))
    state_axes = [n - 1 - qubits[m - 1 - a] for a in range(m)]
    out = np.tensordot(u, t, axes=(col_axes, state_axes))
    # out axes: m row axes (bits m-1..0), then remaining state axes in order
    rest = [ax for ax in range(n) if ax not in state_axes]
    perm_src = state_axes + rest
    inv = np.argsort(perm_src)
    return np.transpose(out, inv).reshape(-1)


def numpy_run(circuit: Circuit, psi0=None) -> np.ndarray:
    n = circuit.n_qubits()
    psi = np.zeros(1 << n, dtype=np.complex128) if psi0 is None else np.array(psi0, dtype=np.complex128)
    if psi0 is None:
        psi[0] = 1.0
    for op in circuit.ops():
        psi = numpy_apply(psi, n, op.gate.matrix, list(op.qubits))
    return psi


def max_abs_diff(a, b) -> float:
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)))) if len(a) else 0.0


def infidelity(a, b) -> float:
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    ov = np.vdot(a, b)
    return float(1.0 - abs(ov) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real))
