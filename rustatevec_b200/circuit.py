"""Circuit representation and fluent builder.

Mirrors qsv's ``circuit.rs`` (crates/qsv-core/src/circuit.rs:13-130): an ordered list of
``GateOp`` (a gate plus the ordered qubits it acts on). ``push`` validates arity, range and
distinctness exactly as ``Circuit::push`` does (circuit.rs:54-78), raising ``ValueError``
where the Rust code panics.

``flatten()`` produces the packed arrays the C ABI (``qsvb_execute``) and the oracle consume:
per-op arity, concatenated qubits, and concatenated row-major interleaved FP64 matrices.
"""
from __future__ import annotations

from dataclasses import dataclass
from itertools import chain
from operator import attrgetter

import numpy as np

from . import gate as G
from .gate import DenseGate, MAX_GATE_QUBITS


_QUBITS = attrgetter("qubits")
_MATRIX = attrgetter("gate.matrix")


def flatten_ops(ops):
    """``(arity u32[nops], qubits u32[sum m], mats f64[sum 2*4^m])`` of a list of ``GateOp``; the
    per-op work runs in C (``map`` + ``attrgetter``, and one ``bytes.join`` over the matrices'
    buffers, which ``DenseGate`` keeps C-contiguous complex128). The matrix array is read-only."""
    if not ops:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32), np.zeros(0, np.float64)
    qs = list(map(_QUBITS, ops))
    arity = np.fromiter(map(len, qs), dtype=np.uint32, count=len(qs))
    qubits = np.fromiter(chain.from_iterable(qs), dtype=np.uint32)
    mats = np.frombuffer(b"".join(map(_MATRIX, ops)), dtype=np.float64)
    return arity, qubits, mats


@dataclass
class GateOp:
    gate: DenseGate
    qubits: tuple

    def n_qubits(self) -> int:
        return len(self.qubits)


class Circuit:
    def __init__(self, n_qubits: int):
        self._n = int(n_qubits)
        self._ops: list[GateOp] = []

    def n_qubits(self) -> int:
        return self._n

    def ops(self) -> list:
        return self._ops

    def __len__(self) -> int:
        return len(self._ops)

    def push(self, g: DenseGate, qubits) -> "Circuit":
        qs = tuple(int(q) for q in qubits)
        if g.n_qubits != len(qs):
            raise ValueError("gate arity must match qubit count")
        if len(qs) > MAX_GATE_QUBITS:
            raise ValueError(f"gates act on at most {MAX_GATE_QUBITS} qubits")
        for q in qs:
            if q < 0 or q >= self._n:
                raise ValueError(f"qubit {q} out of range for {self._n} qubits")
        if len(set(qs)) != len(qs):
            raise ValueError("repeated qubit in gate")
        self._ops.append(GateOp(g, qs))
        return self

    # ---- single-qubit (circuit.rs:81-113)
    def h(self, q): return self.push(G.h(), [q])
    def x(self, q): return self.push(G.x(), [q])
    def y(self, q): return self.push(G.y(), [q])
    def z(self, q): return self.push(G.z(), [q])
    def s(self, q): return self.push(G.s_gate(), [q])
    def t(self, q): return self.push(G.t_gate(), [q])
    def sx(self, q): return self.push(G.sx(), [q])
    def rx(self, q, theta): return self.push(G.rx(theta), [q])
    def ry(self, q, theta): return self.push(G.ry(theta), [q])
    def rz(self, q, theta): return self.push(G.rz(theta), [q])
    def phase(self, q, lam): return self.push(G.phase(lam), [q])

    # ---- two-qubit, control first (circuit.rs:116-130)
    def cx(self, c, t): return self.push(G.cx(), [c, t])
    def cz(self, a, b): return self.push(G.cz(), [a, b])
    def cphase(self, c, t, lam): return self.push(G.cphase(lam), [c, t])
    def swap(self, a, b): return self.push(G.swap(), [a, b])
    def rzz(self, a, b, theta): return self.push(G.rzz(theta), [a, b])

    # ---- packing for the C ABI / oracle
    def flatten(self):
        """Return ``(arity u32[nops], qubits u32[sum m], mats f64[sum 2*4^m])``."""
        return flatten_ops(self._ops)

    @classmethod
    def from_flat(cls, n_qubits, arity, qubits, mats) -> "Circuit":
        c = cls(n_qubits)
        qo = mo = 0
        for m in np.asarray(arity).tolist():
            d = 1 << m
            mat = np.asarray(mats[mo:mo + 2 * d * d], dtype=np.float64).view(np.complex128)
            c.push(DenseGate(m, mat.reshape(d, d).copy()), qubits[qo:qo + m])
            qo += m
            mo += 2 * d * d
        return c
