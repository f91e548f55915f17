"""Gate fusion, ``Circuit -> Circuit`` (crates/qsv-core/src/fusion.rs:26-77).

``fuse(circuit, FusionConfig(max_qubits))`` runs the engine's planner through the C ABI
(``qsvb_fuse``) and needs no GPU. With the default ``planner=PLAN_GREEDY`` the grouping is qsv's
greedy consecutive-only rule (single-gate groups pass through unchanged, multi-gate groups are
composed onto their sorted qubits); composition is FP64. ``PLAN_WINDOW`` additionally lets a gate
join a group across gates on disjoint qubits; ``PLAN_LEARNED`` picks the cheapest plan under the
cost model.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .circuit import Circuit
from .gate import DenseGate


@dataclass
class FusionConfig:
    max_qubits: int = 4  # fusion.rs:31-36 default


def fuse(circuit: Circuit, cfg: FusionConfig = FusionConfig(), planner: int = L.PLAN_GREEDY,
         engine: int = L.ENGINE_AUTO) -> Circuit:
    pc = L.PackedCircuit(circuit)
    opts = L.make_opts(planner, max(1, cfg.max_qubits), engine)
    n = C.c_size_t(0)
    L.check(L.lib().qsvb_fuse(pc.ref(), C.byref(opts), None, C.byref(n), None, 0))
    count = n.value
    gates = (L.Gate * max(count, 1))()
    cap = 2 * 4096 * max(count, 1)
    mats = np.zeros(cap, dtype=np.float64)
    n = C.c_size_t(count)
    L.check(L.lib().qsvb_fuse(pc.ref(), C.byref(opts), gates, C.byref(n), mats.ctypes.data_as(L._dp), cap))
    out = Circuit(circuit.n_qubits())
    mo = 0
    for i in range(n.value):
        g = gates[i]
        m = g.n_qubits
        d = 1 << m
        mat = mats[mo:mo + 2 * d * d].view(np.complex128).reshape(d, d).copy()
        mo += 2 * d * d
        out.push(DenseGate(m, mat), [g.qubits[j] for j in range(m)])
    return out
