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

import numpy as np

from . import gate as G
from .gate import DenseGate, MAX_GATE_QUBITS


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
        arity = np.fromiter((len(op.qubits) for op in self._ops), dtype=np.uint32,
                            count=len(self._ops))
        qubits = np.fromiter((q for op in self._ops for q in op.qubits), dtype=np.uint32)
        if self._ops:
            mats = np.concatenate([op.gate.matrix.reshape(-1).view(np.float64)
                                   for op in self._ops])
        else:
            mats = np.zeros(0, dtype=np.float64)
        return arity, qubits, np.ascontiguousarray(mats)

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
