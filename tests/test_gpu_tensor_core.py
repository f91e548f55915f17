"""Tensor-core (tcgen05, BF16 hi/lo split, FP32 accumulate) dense sweeps vs the FP64 oracle.

Tolerances: one sweep keeps ~16 significant bits per product, so max |d amp| <= 1e-5 holds for
complex64 states, and whole circuits stay within 1-F <= 1e-5 of the FP64 run."""
import math

import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend, Plan, PLAN_AS_GIVEN, PLAN_LEARNED, PLAN_WINDOW, ENGINE_TENSOR_CORE
from rustatevec_b200 import _lib as L
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import brickwork, random_circuit

from helpers import infidelity, max_abs_diff

pytestmark = pytest.mark.gpu


def haar(k, seed):
    rng = np.random.default_rng(seed)
    z = (rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.fixture(scope="module")
def be(built):
    b = B200Backend(0, precision="f32")
    yield b
    b.close()


def run_tc(be, c, psi, planner=PLAN_AS_GIVEN, k=6):
    st = be.alloc(c.n_qubits())
    be.upload(st, psi.real, psi.imag)
    p = Plan(be, c, L.make_opts(planner, k, ENGINE_TENSOR_CORE))
    p.run(st)
    kinds = p.stats()["by_kind"]
    return be.download(st).as_complex(), kinds


QSETS = {
    "high": lambda n, k: list(range(n - k, n)),           # B MN-major (state bits 0-1 are columns)
    "low": lambda n, k: list(range(k)),                   # B K-major (gate owns bits 0-1)
    "mid": lambda n, k: list(range(3, 3 + k)),
    "mixed": lambda n, k: [0] + list(range(5, 4 + k)),    # B row pairs (bit 0 gate, bit 1 column)
    "mixed2": lambda n, k: [1] + list(range(7, 6 + k)),
    # bit 0 a column, bit 1 the gate's lowest qubit, its next qubit state bit 2, 3 or 4 (lane pairs)
    "pair2": lambda n, k: [1, 2] + list(range(8, 6 + k)),
    "pair3": lambda n, k: [1, 3] + list(range(7, 5 + k)),
    "pair4": lambda n, k: [4, 1] + list(range(n - k + 2, n)),
    "spread": lambda n, k: [2, 4, 7, 9, 10, 11][:k],
    "unsorted": lambda n, k: list(reversed(range(n - k, n))),
}


@pytest.mark.parametrize("k", [4, 5, 6])
@pytest.mark.parametrize("qset", sorted(QSETS))
@pytest.mark.parametrize("n", [12, 15])
def test_single_tc_sweep(be, k, qset, n):
    qs = QSETS[qset](n, k)
    psi = random_state(n, 100 * k + n)
    c = Circuit(n)
    c.push(G.DenseGate(k, haar(k, 7 * k + n)), qs)
    got, kinds = run_tc(be, c, psi)
    assert kinds.get("dense_tc", 0) == 1, kinds
    re, im = oracle.run(c, oracle.REF, oracle.F64, state=(psi.real.copy(), psi.imag.copy()))
    want = re + 1j * im
    err = max_abs_diff(want, got)
    assert err < 1e-5, (qset, k, n, err)
    assert infidelity(want, got) < 1e-8


@pytest.mark.parametrize("qs", [
    [5, 6, 11, 12, 13, 14],      # two tile runs -> 2-D tensor-map TMA
    [3, 8, 9, 13, 14, 18],       # four tile runs -> 4-D tensor map
    [5, 6, 11, 12, 17, 18],      # brickwork window shape
    [7, 9, 11, 13, 15, 17],      # seven tile runs -> bulk-copy fallback
    [0, 2, 9, 10, 16, 19],       # bit 0 in the gate, bit 1 a column (scalar B stores)
    [2, 3, 4, 5],                # k = 4, one contiguous tile
    [1, 6, 7, 12, 19],           # k = 5, bit 1 in the gate
    [1, 2, 7, 8, 9, 10],         # brickwork window with bit 1: lane-pair B stores
    [1, 2, 3, 4, 18, 19],        # lane pairs, bits 2-4 all in the gate
    [1, 4, 9, 10, 16],           # k = 5, lane pairs across lane bit 2
    [3, 1, 6, 11],               # k = 4, lane pairs across lane bit 1
])
def test_tc_tile_shapes_n20(be, qs):
    n = 20
    k = len(qs)
    psi = random_state(n, sum(qs))
    c = Circuit(n)
    c.push(G.DenseGate(k, haar(k, 99 + sum(qs))), qs)
    got, kinds = run_tc(be, c, psi)
    assert kinds.get("dense_tc", 0) == 1, kinds
    re, im = oracle.run(c, oracle.CPU_PARALLEL, oracle.F64, state=(psi.real.copy(), psi.imag.copy()))
    want = re + 1j * im
    assert max_abs_diff(want, got) < 1e-5
    assert infidelity(want, got) < 1e-8


@pytest.mark.parametrize("planner", [PLAN_WINDOW, PLAN_LEARNED])
def test_tc_circuits_match_oracle(be, planner):
    for seed in range(6):
        n = 12 + seed % 4
        c = random_circuit(n, 120, 31337 + seed)
        psi = random_state(n, seed)
        got, kinds = run_tc(be, c, psi, planner, 6)
        re, im = oracle.run(c, oracle.REF, oracle.F64, state=(psi.real.copy(), psi.imag.copy()))
        want = re + 1j * im
        assert max_abs_diff(want, got) < 1e-5, (seed, kinds)
        assert infidelity(want, got) < 1e-6


def test_tc_brickwork_fidelity_vs_fp64(be, be64):
    n = 20
    c = brickwork(n, 20, 3)
    st = be.alloc(n)
    be.init_basis(st, 0)
    p = Plan(be, c, L.make_opts(PLAN_LEARNED, 6, ENGINE_TENSOR_CORE))
    p.run(st)
    kinds = p.stats()["by_kind"]
    assert kinds.get("dense_tc", 0) + kinds.get("tc_chain", 0) > 0, kinds
    ref = be64.alloc(n)
    be64.init_basis(ref, 0)
    be64.run(ref, c, L.make_opts(PLAN_AS_GIVEN, 1))
    ip = np.zeros(2)
    L.check(L.lib().qsvb_inner_product(be.ctx, st.handle, ref.handle, ip.ctypes.data_as(L._dp)))
    fid = (ip[0] ** 2 + ip[1] ** 2) / be.norm_sqr(st)
    assert 1.0 - fid < 1e-5, 1.0 - fid
