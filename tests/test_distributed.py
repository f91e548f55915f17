"""A state spread over 2^g ranks (host logic, CPU): the global-qubit planner and the block
exchange, with the oracle as each rank's local engine. Checked against the oracle's run of the
whole circuit on one state, in one process (every rank a slice) and over world-size-2 and -4 gloo
groups (one rank per process)."""
import contextlib
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

import oracle
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import brickwork, ghz_chain, qaoa_maxcut, qft, random_circuit
from rustatevec_b200.distributed import (DistributedState, ExchangeStep, LocalStep, Layout, TorchComm,
                                         plan_cost, plan_distributed, rank_circuit)


class OracleSliceEngine:
    """Each rank's slice as FP64 numpy arrays run by the oracle (test stand-in for the CUDA engine)."""

    def alloc(self, nl):
        return [np.zeros(1 << nl), np.zeros(1 << nl)]

    def views(self, st):
        return torch.from_numpy(st[0]), torch.from_numpy(st[1])

    def stream(self):
        return contextlib.nullcontext()

    def init_basis(self, st, basis):
        st[0][:] = 0
        st[1][:] = 0
        if basis is not None:
            st[0][basis] = 1.0

    def run(self, st, circuit):
        if len(circuit):
            re, im = oracle.run(circuit, oracle.REF, oracle.F64, state=(st[0], st[1]))
            st[0][:] = re
            st[1][:] = im

    def expectation_z(self, st, mask):
        p = st[0] ** 2 + st[1] ** 2
        return oracle.expectation_z(p, mask)

    def download(self, st):
        return st[0].copy(), st[1].copy()


def whole(c):
    re, im = oracle.run(c, oracle.REF, oracle.F64)
    return re + 1j * im


def circuits(n):
    c = Circuit(n)
    for q in range(n):
        c.h(q)
    c.cx(n - 1, 0).cz(n - 2, n - 1).cphase(n - 1, 1, 0.3).rzz(n - 3, n - 1, 0.7)
    c.push(G.controlled_1q(G.ry(0.4)), [n - 1, n - 2])   # control and target both global for g >= 2
    c.swap(0, n - 1)
    return [random_circuit(n, 12 * n, 3 + n), qft(n), brickwork(n, 4, n), ghz_chain(n), qaoa_maxcut(n, 2, n), c]


@pytest.mark.parametrize("g", [1, 2, 3])
def test_slices_in_one_process_match_the_whole_state(built, g):
    for n in (9, 11):
        for c in circuits(n):
            ds = DistributedState(n, g, OracleSliceEngine())
            ds.init_basis(0)
            ds.run(c)
            got = ds.gather()
            assert np.max(np.abs(got - whole(c))) < 1e-12
            assert abs(ds.norm_sqr() - 1) < 1e-12
            p = np.abs(whole(c)) ** 2
            for mask in (1, 1 << (n - 1), (1 << n) - 1, 0b1011):
                assert abs(ds.expectation_z(mask) - oracle.expectation_z(p, mask)) < 1e-12


def test_runs_continue_from_the_moved_layout_and_basis_inputs(built):
    n, g = 10, 2
    a, b = random_circuit(n, 60, 1), qft(n)
    ds = DistributedState(n, g, OracleSliceEngine())
    ds.init_basis(0b1010010011)
    ds.run(a)
    ds.run(b)
    ab = Circuit(n)
    ab.ops().extend(a.ops())
    ab.ops().extend(b.ops())
    re, im = oracle.run(ab, oracle.REF, oracle.F64,
                        state=(np.eye(1 << n)[0b1010010011], np.zeros(1 << n)))
    assert np.max(np.abs(ds.gather() - (re + 1j * im))) < 1e-12


def test_non_mixing_gates_on_global_qubits_need_no_exchange(built):
    n, g = 10, 3
    c = Circuit(n)
    for q in range(n):
        c.rz(q, 0.1 * q)
    for q in range(n - 1):
        c.cz(q, q + 1).rzz(q, n - 1, 0.2).cphase(n - 1, n - 2, 0.5)
    c.cx(n - 1, 0)  # control global, target local: block-diagonal in the control
    steps, lay = plan_distributed(c, g)
    assert not any(isinstance(s, ExchangeStep) for s in steps)
    assert lay.phys == list(range(n))


def test_exchange_steps_use_the_top_local_positions_and_the_gate_is_local_after(built):
    n, g = 12, 3
    c = random_circuit(n, 200, 9)
    steps, _ = plan_distributed(c, g)
    nl = n - g
    lay = Layout(n, g)
    for s in steps:
        if isinstance(s, ExchangeStep):
            assert sorted(s.tpos) == list(range(nl - len(s.gbits), nl))
            assert len(set(s.gbits)) == len(s.gbits)
            for gb, t in zip(s.gbits, s.tpos):
                lay.swap_positions(nl + gb, t)
        else:
            for op in s.ops:
                if op.matrix.shape[0] == 4 and np.array_equal(op.matrix, G.swap().matrix) and not op.glob:
                    lay.swap_positions(op.local[0][1], op.local[1][1])
    assert sum(isinstance(s, ExchangeStep) for s in steps) > 0


def test_rank_circuits_fix_the_global_bits():
    # CX with its control global: ranks with the bit set apply X, the others nothing
    c = Circuit(8).cx(7, 0)
    steps, _ = plan_distributed(c, 1)
    assert len(steps) == 1 and isinstance(steps[0], LocalStep)
    assert len(rank_circuit(steps[0], 7, 0)) == 0
    r1 = rank_circuit(steps[0], 7, 1)
    assert len(r1) == 1 and np.array_equal(r1.ops()[0].gate.matrix, G.x().matrix)
    # CZ on two global qubits: a -1 phase on the rank whose bits are both set
    c = Circuit(9).cz(7, 8)
    steps, _ = plan_distributed(c, 2)
    assert [len(rank_circuit(steps[0], 7, r)) for r in range(4)] == [0, 0, 0, 1]
    assert np.allclose(rank_circuit(steps[0], 7, 3).ops()[0].gate.matrix, -np.eye(2))


def test_auto_policy_keeps_the_cheaper_plan():
    # brickwork uses every qubit every layer: moving victims by SWAP costs more than it saves;
    # QAOA's mixers and cost layers reuse qubits unevenly: furthest-next-use wins
    for c, g in ((brickwork(16, 8, 1), 1), (qaoa_maxcut(16, 3, 2), 1), (qft(14), 2), (random_circuit(14, 200, 7), 2)):
        costs = [plan_cost(plan_distributed(c, g, policy=p, group=grp)[0])
                 for p in ("furthest", "top") for grp in (False, True)]
        auto = plan_cost(plan_distributed(c, g, policy="auto")[0])
        assert auto == min(costs)
    with pytest.raises(ValueError):
        plan_distributed(Circuit(8), 1, policy="nearest")


@pytest.mark.parametrize("policy", ["furthest", "top", "furthest+group", "top+group"])
def test_every_policy_matches_the_whole_state(built, policy):
    n, g = 10, 3
    for c in circuits(n):
        ds = DistributedState(n, g, OracleSliceEngine(), policy=policy)
        ds.init_basis(0)
        ds.run(c)
        assert np.max(np.abs(ds.gather() - whole(c))) < 1e-12


def test_rejects_too_few_local_qubits():
    with pytest.raises(ValueError):
        plan_distributed(Circuit(7), 2)
    with pytest.raises(ValueError):
        DistributedState(7, 2, OracleSliceEngine())


def _worker(rank, world, port, g, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n = 10
        res = []
        for c in circuits(n):
            ds = DistributedState(n, g, OracleSliceEngine(), TorchComm(), chunk_elems=37)
            ds.init_basis(0)
            st = ds.run(c)
            got = ds.gather()
            z = ds.expectation_z((1 << n) - 1)
            res.append((got, z, st["exchanges"]))
        out[rank] = res
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("g", [1, 2])
def test_gloo_ranks_match_the_whole_state(built, g):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 1 << g
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, g, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    n = 10
    for i, c in enumerate(circuits(n)):
        want = whole(c)
        got, z, ex = out[0][i]
        assert np.max(np.abs(got - want)) < 1e-12
        zw = oracle.expectation_z(np.abs(want) ** 2, (1 << n) - 1)
        for r in range(world):
            assert abs(out[r][i][1] - zw) < 1e-12
            assert out[r][i][2] == ex
            if r:
                assert out[r][i][0] is None


def test_random_circuits_every_policy_property(built):
    """Property check over seeded random cases: any width, global-bit count, policy and grouping
    gives the oracle's whole-state result."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=40, deadline=None, derandomize=True)
    @given(n=st.integers(8, 11), g=st.integers(1, 3), depth=st.integers(5, 60), seed=st.integers(0, 10 ** 6),
           policy=st.sampled_from(["auto", "furthest", "top", "furthest+group", "top+group"]))
    def check(n, g, depth, seed, policy):
        if n - g < 6:
            return
        c = random_circuit(n, depth, seed)
        ds = DistributedState(n, g, OracleSliceEngine(), policy=policy, chunk_elems=1 + seed % 300)
        ds.init_basis(seed % (1 << n))
        ds.run(c)
        psi0 = np.zeros(1 << n)
        psi0[seed % (1 << n)] = 1.0
        re, im = oracle.run(c, oracle.REF, oracle.F64, state=(psi0, np.zeros(1 << n)))
        assert np.max(np.abs(ds.gather() - (re + 1j * im))) < 1e-12

    check()
