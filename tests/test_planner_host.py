"""Planner decisions on the host (no device): qsvb_plan_dry_run plans a circuit exactly as
qsvb_execute would and reports the sweeps by kind."""
import ctypes as C

import pytest

from rustatevec_b200 import _lib as L
from rustatevec_b200 import tuning
from rustatevec_b200.circuits import brickwork, ghz_chain, qaoa_maxcut, qft, random_circuit


def dry(circ, planner, k=4, dtype=L.C64, engine=L.ENGINE_AUTO):
    st = L.PlanStats()
    pc = L.PackedCircuit(circ)  # owns the gate structs and matrices for the duration of the call
    L.check(L.lib().qsvb_plan_dry_run(pc.ref(), dtype, C.byref(L.make_opts(planner, k, engine)), C.byref(st)))
    return st.to_dict()


def test_tile_planner_passes(built):
    # QFT(32): the Hadamards of blocks of qubits plus every controlled phase (diagonals may reach
    # outside the tile) in a handful of passes, then the final swaps
    st = dry(qft(32), L.PLAN_TILE)
    assert set(st["by_kind"]) == {"tile"} and st["n_sweeps"] <= 8
    st = dry(ghz_chain(24), L.PLAN_TILE, dtype=L.C128)
    assert set(st["by_kind"]) == {"tile"} and st["n_sweeps"] <= 4
    # too small for tiles: ordinary sweeps
    assert "tile" not in dry(random_circuit(12, 80, 1), L.PLAN_TILE)["by_kind"]


def test_wide_gates_stay_fused_sweeps(built):
    from rustatevec_b200 import DenseGate
    import numpy as np
    c = random_circuit(20, 60, 3)
    c.push(DenseGate(3, np.eye(8, dtype=complex) * 1j), [1, 7, 19])
    for op in random_circuit(20, 60, 4).ops():
        c.push(op.gate, op.qubits)
    st = dry(c, L.PLAN_TILE)
    assert st["by_kind"].get("tile", 0) >= 2 and sum(v for k, v in st["by_kind"].items() if k != "tile") >= 1


def test_learned_planner_choices_with_the_trained_model(built):
    doc = tuning.load()
    if doc is None:
        pytest.skip("no trained model in the tree")
    try:
        st = dry(brickwork(30, 20, 0), L.PLAN_LEARNED, 6)
        # k>=5 blocks on tensor cores, as single-matrix sweeps or chained passes
        assert st["by_kind"].get("dense_tc", 0) >= 40 or st["by_kind"].get("tc_chain", 0) >= 20, st
        assert dry(brickwork(30, 20, 0), L.PLAN_LEARNED, 6, engine=L.ENGINE_CUDA_CORE)["by_kind"].get("dense_tc", 0) == 0
        q = dry(qaoa_maxcut(33, 4, 0), L.PLAN_LEARNED, 6, dtype=L.C128)
        g = dry(qaoa_maxcut(33, 4, 0), L.PLAN_GREEDY, 4, dtype=L.C128)
        assert q["predicted_seconds"] < g["predicted_seconds"] and q["n_sweeps"] < g["n_sweeps"]
    finally:
        tuning.install(None)


def test_predictions_above_the_trained_size_respect_the_memory_floor(built):
    """The cost model is trained on states of at most 30 qubits; larger states are predicted as the
    same sweep on a 30-qubit state times the amplitude ratio, so no plan is predicted faster than
    its algorithmic bytes at the measured copy bandwidth (about 6.55 TB/s)."""
    doc = tuning.load()
    if doc is None:
        pytest.skip("no trained model in the tree")
    try:
        for circ, dtype in ((qaoa_maxcut(33, 4, 0), L.C128), (qaoa_maxcut(31, 2, 0), L.C128),
                            (qft(32), L.C64), (brickwork(32, 6, 0), L.C64)):
            for planner, k in ((L.PLAN_GREEDY, 4), (L.PLAN_WINDOW, 5), (L.PLAN_LEARNED, 6)):
                st = dry(circ, planner, k, dtype=dtype)
                assert st["predicted_seconds"] >= st["algorithmic_bytes"] / 6.6e12, (circ.n_qubits(), planner)
    finally:
        tuning.install(None)


def test_dry_run_rejects_bad_input(built):
    st = L.PlanStats()
    assert L.lib().qsvb_plan_dry_run(None, 0, None, C.byref(st)) == L.QSVB_E_INVALID
    pc = L.PackedCircuit(qft(4))
    assert L.lib().qsvb_plan_dry_run(pc.ref(), 7, None, C.byref(st)) == L.QSVB_E_INVALID


def test_chain_planner_passes(built):
    """PLAN_CHAIN: brickwork 30q depth 20 in far fewer passes than one sweep per fused 6-qubit
    block; the layout is restored by a few permutation passes; other states plan as WINDOW.
    The pass counts are those of the current planner (qubits bound for a tile's high side go to
    their own state bit when it is free): 63 + 3, 37 + 2 and 27 + 3 chain + permutation passes
    at one, two and three matrices a pass."""
    c = brickwork(30, 20, 0)
    win = dry(c, L.PLAN_WINDOW, 6)
    for mats, most, perm in ((1, 63, 3), (2, 37, 2), (3, 27, 3)):
        st = L.PlanStats()
        pc = L.PackedCircuit(c)
        o = L.make_opts(L.PLAN_CHAIN, 6, L.ENGINE_AUTO, chain_max_matrices=mats)
        L.check(L.lib().qsvb_plan_dry_run(pc.ref(), L.C64, C.byref(o), C.byref(st)))
        d = st.to_dict()
        assert set(d["by_kind"]) <= {"tc_chain", "permute"}, d
        assert d["by_kind"]["tc_chain"] <= most and d["by_kind"].get("permute", 0) <= perm, d
        assert d["n_sweeps"] < win["n_sweeps"] or mats == 1
    assert "tc_chain" not in dry(c, L.PLAN_CHAIN, 6, dtype=L.C128)["by_kind"]
    assert "tc_chain" not in dry(random_circuit(11, 60, 1), L.PLAN_CHAIN, 6)["by_kind"]
    assert "tc_chain" not in dry(c, L.PLAN_CHAIN, 6, engine=L.ENGINE_CUDA_CORE)["by_kind"]
