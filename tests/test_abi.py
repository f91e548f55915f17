"""The C-ABI library: loads, exports every symbol include/qsvb.h declares, and validates input
on the host (no GPU needed for these)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from rustatevec_b200 import _lib as L
from rustatevec_b200 import FusionConfig, fuse, PLAN_GREEDY, PLAN_WINDOW, PLAN_LEARNED, PLAN_AS_GIVEN
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import brickwork, qft, random_circuit, qaoa_maxcut

from helpers import max_abs_diff

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            out |= set(re.findall(r"^\s*(?:int|const char\*|void)\s+(qsvb_\w+)\s*\(", txt, re.M))
    return out


def test_library_exports_every_declared_symbol(built):
    lib = L.lib()
    syms = declared_symbols()
    assert len(syms) >= 25
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert lib.qsvb_version().decode().startswith("qsvb")


def test_python_signatures_cover_the_header(built):
    assert declared_symbols() <= set(L.SIGNATURES)


def test_greedy_fuse_matches_oracle_fuse(built):
    # the engine's GREEDY planner is the reference fuse (fusion.rs:39-140), composed in FP64
    for mq in (2, 3, 4, 5, 6):
        for seed in range(20):
            n = 4 + seed % 5
            c = random_circuit(n, 50, 70000 + seed)
            ours = fuse(c, FusionConfig(mq)).flatten()
            theirs = oracle.fuse(c, mq, oracle.F64)
            assert np.array_equal(ours[0], theirs[0]) and np.array_equal(ours[1], theirs[1])
            assert max_abs_diff(ours[2], theirs[2]) < 1e-13


@pytest.mark.parametrize("planner", [PLAN_WINDOW, PLAN_LEARNED])
def test_reordering_planners_are_exact(built, planner):
    for mq in (2, 4, 6):
        for seed in range(15):
            n = 4 + seed % 5
            c = random_circuit(n, 60, 123 + seed)
            f = fuse(c, FusionConfig(mq), planner=planner)
            assert len(f) <= len(c)
            a, b = oracle.run(c), oracle.run(f)
            assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < 1e-12
    c = qft(7)
    f = fuse(c, FusionConfig(5), planner=planner)
    a, b = oracle.run(c), oracle.run(f)
    assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < 1e-12


def test_window_fusion_beats_greedy_on_brickwork(built):
    c = brickwork(30, 20, 0)
    for k in (4, 5, 6):
        assert len(fuse(c, FusionConfig(k), planner=PLAN_WINDOW)) < len(fuse(c, FusionConfig(k)))


def test_as_given_is_identity(built):
    c = random_circuit(6, 30, 5)
    f = fuse(c, FusionConfig(4), planner=PLAN_AS_GIVEN)
    assert np.array_equal(f.flatten()[2], c.flatten()[2])


def bad_call(circuit_struct):
    n = C.c_size_t(0)
    return L.lib().qsvb_fuse(C.byref(circuit_struct), None, None, C.byref(n), None, 0)


def test_invalid_circuits_are_rejected_with_a_message(built):
    mat = np.eye(4, dtype=np.complex128).reshape(-1).view(np.float64).copy()
    g = L.Gate()
    g.n_qubits = 2
    g.qubits[0], g.qubits[1] = 0, 0  # repeated qubit
    g.matrix = mat.ctypes.data_as(L._dp)
    arr = (L.Gate * 1)(g)
    cs = L.CircuitS(3, 1, C.cast(arr, C.POINTER(L.Gate)))
    assert bad_call(cs) == L.QSVB_E_INVALID
    assert "repeated qubit" in L.lib().qsvb_last_error().decode()
    arr[0].qubits[1] = 7  # out of range
    assert bad_call(cs) == L.QSVB_E_INVALID
    assert "out of range" in L.lib().qsvb_last_error().decode()
    arr[0].qubits[1] = 1
    arr[0].n_qubits = 7  # arity
    assert bad_call(cs) == L.QSVB_E_INVALID
    arr[0].n_qubits = 2
    arr[0].matrix = None
    assert bad_call(cs) == L.QSVB_E_INVALID
    assert L.lib().qsvb_fuse(None, None, None, None, None, 0) == L.QSVB_E_INVALID


def test_null_handles_fail_cleanly(built):
    lib = L.lib()
    out = C.c_double()
    assert lib.qsvb_norm_sqr(None, None, C.byref(out)) == L.QSVB_E_INVALID
    assert lib.qsvb_destroy(None) == L.QSVB_OK
    assert lib.qsvb_state_info(None, None, None, None, None) == L.QSVB_E_INVALID


def test_qaoa_generator_graph_rule():
    from rustatevec_b200.circuits import regular_graph
    e = regular_graph(33, 7)
    deg = np.zeros(33, int)
    for a, b in e:
        assert a != b
        deg[a] += 1
        deg[b] += 1
    assert deg[0] == 4 and np.all(deg[1:] == 3) and len(set(e)) == len(e) == 50
    c = qaoa_maxcut(12, 2, 3)
    assert c.n_qubits() == 12


def test_packed_batch_matches_per_circuit_packing():
    """The numpy-built batch packing lays out the same gate structs as PackedCircuit."""
    import ctypes as C
    from rustatevec_b200.circuits import ansatz_batch, random_circuit
    circuits = ansatz_batch(5, 1, n_lo=3, n_hi=9, d_lo=1, d_hi=3) + [random_circuit(6, 40, 3)]
    pb = L.PackedBatch(circuits)
    assert pb.count == len(circuits)
    for i, circ in enumerate(circuits):
        pc = L.PackedCircuit(circ)
        row = pb.circs[i]
        assert int(row["n"]) == circ.n_qubits() and int(row["ngates"]) == pc.struct.n_gates
        g = np.frombuffer((C.c_char * (40 * pc.struct.n_gates)).from_address(int(row["gates"])), dtype=L._GATE_DT)
        for k in range(pc.struct.n_gates):
            a = pc.gates[k]
            m = a.n_qubits
            assert int(g[k]["n"]) == m and list(a.qubits)[:m] == [int(x) for x in g[k]["q"][:m]]
            want = np.ctypeslib.as_array(a.matrix, shape=(2 << (2 * m),))
            got = np.ctypeslib.as_array(C.cast(int(g[k]["mat"]), C.POINTER(C.c_double)), shape=(2 << (2 * m),))
            assert np.array_equal(want, got)
