"""Gate representation and the standard gate library.

Mirrors qsv's ``gate.rs`` (crates/qsv-core/src/gate.rs:19-180): a ``DenseGate`` is a
``2^m x 2^m`` complex matrix stored row-major. Matrices are always held in FP64 here
(``complex128``); a complex64 circuit rounds them to f32 at the device boundary, the same
rounding ``Cplx::from_f64`` performs (crates/qsv-core/src/complex.rs:45-50).

Qubit convention (gate.rs:8-13): bit ``j`` (LSB = 0) of the gate's row/column index is the
state bit ``qubits[j]``; controlled gates put the control first, so ``cx(c, t)`` acts on
``[c, t]`` with internal index ``bit_c + 2*bit_t``.
"""
from __future__ import annotations

import math

import numpy as np

MAX_GATE_QUBITS = 6


class DenseGate:
    """A dense ``2^m x 2^m`` unitary (gate.rs:19-50)."""

    __slots__ = ("matrix", "n_qubits")

    def __init__(self, n_qubits: int, matrix):
        mat = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
        dim = 1 << n_qubits
        if mat.shape != (dim, dim):
            raise ValueError(f"gate matrix must be {dim}x{dim}, got {mat.shape}")
        self.n_qubits = int(n_qubits)
        self.matrix = mat

    def dim(self) -> int:
        return 1 << self.n_qubits

    def at(self, row: int, col: int) -> complex:
        return complex(self.matrix[row, col])

    def is_diagonal(self) -> bool:
        """Exact-zero off-diagonal test (gate.rs:56-68)."""
        off = self.matrix - np.diag(np.diag(self.matrix))
        return not np.any(off != 0)

    def __repr__(self) -> str:
        return f"DenseGate(n_qubits={self.n_qubits})"


def _g(rows) -> DenseGate:
    m = np.array(rows, dtype=np.complex128)
    return DenseGate(int(round(math.log2(m.shape[0]))), m)


def controlled_1q(u: DenseGate) -> DenseGate:
    """Wrap a 1-qubit gate as ``[control, target]`` (gate.rs:72-87)."""
    if u.n_qubits != 1:
        raise ValueError("controlled_1q needs a 1-qubit gate")
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = 1.0
    m[2, 2] = 1.0
    for to in range(2):
        for ti in range(2):
            m[1 + 2 * to, 1 + 2 * ti] = u.matrix[to, ti]
    return DenseGate(2, m)


_R2 = 0.70710678118654752440  # FRAC_1_SQRT_2


def h():
    return _g([[_R2, _R2], [_R2, -_R2]])


def x():
    return _g([[0, 1], [1, 0]])


def y():
    return _g([[0, -1j], [1j, 0]])


def z():
    return _g([[1, 0], [0, -1]])


def s_gate():
    return _g([[1, 0], [0, 1j]])


def t_gate():
    return _g([[1, 0], [0, complex(_R2, _R2)]])


def sx():
    return _g([[0.5 + 0.5j, 0.5 - 0.5j], [0.5 - 0.5j, 0.5 + 0.5j]])


def rx(theta: float):
    s, c = math.sin(theta * 0.5), math.cos(theta * 0.5)
    return _g([[c, -1j * s], [-1j * s, c]])


def ry(theta: float):
    s, c = math.sin(theta * 0.5), math.cos(theta * 0.5)
    return _g([[c, -s], [s, c]])


def rz(theta: float):
    """``diag(e^{-i theta/2}, e^{+i theta/2})`` (gate.rs:134-138)."""
    s, c = math.sin(theta * 0.5), math.cos(theta * 0.5)
    return _g([[complex(c, -s), 0], [0, complex(c, s)]])


def phase(lam: float):
    s, c = math.sin(lam), math.cos(lam)
    return _g([[1, 0], [0, complex(c, s)]])


def cx():
    return controlled_1q(x())


def cz():
    return controlled_1q(z())


def cphase(lam: float):
    return controlled_1q(phase(lam))


def swap():
    m = np.zeros((4, 4), dtype=np.complex128)
    m[0, 0] = m[1, 2] = m[2, 1] = m[3, 3] = 1.0
    return DenseGate(2, m)


def rzz(theta: float):
    """``exp(-i theta/2 Z(x)Z)`` on ``[a, b]`` (gate.rs:170-180)."""
    m = np.zeros((4, 4), dtype=np.complex128)
    for idx in range(4):
        parity = (idx & 1) ^ ((idx >> 1) & 1)
        zz = 1.0 if parity == 0 else -1.0
        a = -0.5 * theta * zz
        m[idx, idx] = complex(math.cos(a), math.sin(a))
    return DenseGate(2, m)


def u_from_quaternion(a: float, b: float, c: float, d: float):
    """SU(2) element ``[[a+ib, c+id], [-c+id, a-ib]]`` of a unit quaternion (a, b, c, d)."""
    return _g([[complex(a, b), complex(c, d)], [complex(-c, d), complex(a, -b)]])


LIBRARY = {
    "h": h, "x": x, "y": y, "z": z, "s": s_gate, "t": t_gate, "sx": sx,
    "rx": rx, "ry": ry, "rz": rz, "phase": phase,
    "cx": cx, "cz": cz, "cphase": cphase, "swap": swap, "rzz": rzz,
}
PARAMETRIC = {"rx", "ry", "rz", "phase", "cphase", "rzz"}
