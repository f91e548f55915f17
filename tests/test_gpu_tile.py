"""Tile sweeps (QSVB_PLAN_TILE, and the learned planner when it picks them): runs of 1- and
2-qubit gates applied on shared-memory tiles, against the oracle (RefBackend restatement,
crates/qsv-core/src/backend/reference.rs:35-62) on the same circuits and inputs."""
import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend, DenseGate, PLAN_LEARNED, PLAN_TILE, ENGINE_AUTO
from rustatevec_b200 import _lib as L
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import brickwork, ghz_chain, qaoa_maxcut, qft, random_circuit

from helpers import max_abs_diff

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def ref_state(c, psi0=None):
    if psi0 is None:
        re, im = oracle.run(c, oracle.REF, oracle.F64)
    else:
        re, im = oracle.run(c, oracle.REF, oracle.F64, state=(psi0.real.copy(), psi0.imag.copy()))
    return re + 1j * im


def run(be, c, planner=PLAN_TILE, psi0=None):
    st = be.alloc(c.n_qubits())
    if psi0 is None:
        be.init_basis(st, 0)
    else:
        be.upload(st, psi0.real, psi0.imag)
    stats = be.run(st, c, L.make_opts(planner, 4, ENGINE_AUTO))
    out = be.download(st).as_complex()
    st.free()
    return out, stats


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("n", [15, 17, 20])
def test_random_circuits(be, n):
    c = random_circuit(n, 12 * n, 0x7117 + n)
    got, st = run(be, c)
    assert st["by_kind"].get("tile", 0) >= 1
    assert max_abs_diff(ref_state(c), got) < TOL[be.precision]


def test_arbitrary_input_state_and_wide_local_sets(be):
    n = 22
    c = random_circuit(n, 300, 99)
    psi = random_state(n, 5)
    got, st = run(be, c, psi0=psi)
    assert st["by_kind"].get("tile", 0) >= 1
    assert max_abs_diff(ref_state(c, psi), got) < TOL[be.precision]


def test_qft_on_gaussian_state(be):
    n = 18
    psi = random_state(n, 11)
    c = qft(n)
    for planner in (PLAN_TILE, PLAN_LEARNED):
        got, _ = run(be, c, planner, psi)
        assert max_abs_diff(ref_state(c, psi), got) < TOL[be.precision], planner


def test_qaoa_and_brickwork(be):
    for c in (qaoa_maxcut(17, 2, 3), brickwork(16, 6, 2)):
        for planner in (PLAN_TILE, PLAN_LEARNED):
            got, _ = run(be, c, planner)
            assert max_abs_diff(ref_state(c), got) < TOL[be.precision], (c.n_qubits(), planner)


def test_ghz_chain_known_answer(be):
    n = 20
    got, st = run(be, ghz_chain(n))
    p = np.abs(got) ** 2
    assert abs(p[0] - 0.5) < TOL[be.precision] and abs(p[-1] - 0.5) < TOL[be.precision]
    assert abs(p.sum() - 1.0) < TOL[be.precision]


def test_wider_gates_split_tile_runs(be):
    n = 16
    c = random_circuit(n, 100, 4)
    rng = np.random.default_rng(2)
    z = rng.normal(size=(8, 8)) + 1j * rng.normal(size=(8, 8))
    q, _ = np.linalg.qr(z)
    c.push(DenseGate(3, q), [2, 9, 15])
    for op in random_circuit(n, 100, 5).ops():
        c.push(op.gate, op.qubits)
    got, st = run(be, c)
    assert st["by_kind"].get("tile", 0) >= 2 and st["by_kind"].get("dense", 0) + st["by_kind"].get("dense_tc", 0) >= 1
    assert max_abs_diff(ref_state(c), got) < TOL[be.precision]


def test_small_states_use_ordinary_sweeps(be):
    c = random_circuit(10, 60, 1)
    got, st = run(be, c)
    assert "tile" not in st["by_kind"]
    assert max_abs_diff(ref_state(c), got) < TOL[be.precision]


def test_diagonals_reaching_outside_the_tile(be):
    """Diagonal gates whose qubits lie outside a pass's local set ride along as per-tile phases:
    one qubit outside (either gate position), both outside, and 1-qubit phases outside."""
    import math
    n = 21
    c = Circuit(n)
    rng = np.random.default_rng(8)
    for layer in range(3):
        for q in range(n):
            c.h(q) if (q + layer) % 3 else c.rx(q, 0.3 + q)
        for _ in range(40):
            a, b = rng.choice(n, size=2, replace=False)
            kind = rng.integers(4)
            if kind == 0:
                c.cphase(int(a), int(b), float(rng.uniform(0, 2 * math.pi)))
            elif kind == 1:
                c.cz(int(a), int(b))
            elif kind == 2:
                c.rzz(int(a), int(b), float(rng.uniform(0, 2 * math.pi)))
            else:
                c.rz(int(a), float(rng.uniform(0, 2 * math.pi)))
    psi = random_state(n, 21)
    got, st = run(be, c, psi0=psi)
    assert st["by_kind"].get("tile", 0) >= 1
    assert max_abs_diff(ref_state(c, psi), got) < TOL[be.precision]
