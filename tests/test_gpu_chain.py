"""Tensor-core chain passes (PLAN_CHAIN): up to three fused 6-qubit matrices per pass on tcgen05
(bf16 hi/lo split, FP32 accumulate) over 4096-amplitude tiles, each pass relabelling which qubits
sit on the state's low bits, and permutation passes that put every qubit back on its own bit.

Bars, as for every tensor-core path: max |d amp| <= 1e-5 against the FP64 oracle on the same
input, and 1-F <= 1e-5."""
import math

import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend, Plan, PLAN_CHAIN
from rustatevec_b200 import _lib as L
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import brickwork, qft, random_circuit

from helpers import infidelity, max_abs_diff

pytestmark = pytest.mark.gpu


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def haar(k, seed):
    rng = np.random.default_rng(seed)
    z = (rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.fixture(scope="module")
def be(built):
    b = B200Backend(0, precision="f32")
    yield b
    b.close()


def run_chain(be, c, psi, mats=0):
    st = be.alloc(c.n_qubits())
    be.upload(st, psi.real, psi.imag)
    p = Plan(be, c, L.make_opts(PLAN_CHAIN, 6, L.ENGINE_AUTO, chain_max_matrices=mats))
    p.run(st)
    out = be.download(st).as_complex()
    kinds = p.stats()["by_kind"]
    st.free()
    p.free()
    return out, kinds


def check(c, psi, got):
    re, im = oracle.run(c, oracle.CPU_PARALLEL, oracle.F64, state=(psi.real.copy(), psi.imag.copy()))
    want = re + 1j * im
    err = max_abs_diff(want, got)
    inf = infidelity(want, got)
    assert err < 1e-5, err
    assert inf < 1e-5, inf
    return err, inf


@pytest.mark.parametrize("mats", [1, 2, 3])
@pytest.mark.parametrize("n", [12, 13, 16])
def test_chain_random_circuits(be, n, mats):
    c = random_circuit(n, 12 * n, 500 + 10 * n + mats)
    psi = random_state(n, n + mats)
    got, kinds = run_chain(be, c, psi, mats)
    assert kinds.get("tc_chain", 0) >= 1, kinds
    check(c, psi, got)


@pytest.mark.parametrize("mats", [2, 3])
def test_chain_brickwork_many_tiles_per_block(be, mats):
    # 2^20 amplitudes: 256 tiles over the persistent grid, so blocks take several waves of tiles
    n = 20
    c = brickwork(n, 12, 7)
    psi = random_state(n, 20 + mats)
    got, kinds = run_chain(be, c, psi, mats)
    assert kinds.get("tc_chain", 0) >= 3 and kinds.get("permute", 0) >= 1, kinds
    check(c, psi, got)


@pytest.mark.parametrize("first", [
    [0, 1, 2, 3, 4, 5],        # state bits 0, 1 are rows: K-major vectors
    [6, 7, 8, 9, 10, 11],      # bits 0, 1 columns: MN-major
    [0, 7, 8, 9, 10, 13],      # bit 0 a row, bit 1 a column: row pairs
    [1, 2, 9, 10, 12, 13],     # bit 1 row 0, bit 2 row 1: lane pairs
    [1, 4, 7, 8, 9, 14],       # lane pairs across lane bit 2
])
def test_chain_first_matrix_layouts(be, first):
    # the first matrix of the first pass is a Haar 6-qubit unitary on `first`; two more follow
    n = 15
    c = Circuit(n)
    c.push(G.DenseGate(6, haar(6, sum(first))), first)
    c.push(G.DenseGate(6, haar(6, 3 + sum(first))), [2, 3, 5, 8, 11, 14])
    c.push(G.DenseGate(6, haar(6, 5 + sum(first))), [0, 1, 4, 6, 7, 12])
    psi = random_state(n, sum(first))
    got, kinds = run_chain(be, c, psi, 3)
    check(c, psi, got)


def test_chain_qft_and_permutation_passes(be):
    n = 14
    c = qft(n)
    psi = random_state(n, 3)
    got, kinds = run_chain(be, c, psi, 3)
    check(c, psi, got)


def test_chain_brickwork_fidelity_vs_fp64_at_24_qubits(be, be64):
    n = 24
    c = brickwork(n, 20, 3)
    st = be.alloc(n)
    be.init_basis(st, 0)
    p = Plan(be, c, L.make_opts(PLAN_CHAIN, 6, L.ENGINE_AUTO, chain_max_matrices=3))
    p.run(st)
    assert p.stats()["by_kind"].get("tc_chain", 0) > 0
    ref = be64.alloc(n)
    be64.init_basis(ref, 0)
    be64.run(ref, c, L.make_opts(L.PLAN_AS_GIVEN, 1))
    ip = np.zeros(2)
    L.check(L.lib().qsvb_inner_product(be.ctx, st.handle, ref.handle, ip.ctypes.data_as(L._dp)))
    fid = (ip[0] ** 2 + ip[1] ** 2) / be.norm_sqr(st)
    assert 1.0 - fid < 1e-5, 1.0 - fid
    st.free()
    ref.free()
    p.free()


def test_chain_plan_replays_are_deterministic(be):
    n = 16
    c = brickwork(n, 10, 11)
    st = be.alloc(n)
    p = Plan(be, c, L.make_opts(PLAN_CHAIN, 6, L.ENGINE_AUTO, chain_max_matrices=3))
    outs = []
    for _ in range(3):
        be.init_basis(st, 0)
        p.run(st)
        outs.append(be.download(st).as_complex())
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
    st.free()
    p.free()
