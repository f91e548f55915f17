"""Sharding of independent circuits over ranks (host logic, CPU): the LPT split, and the gather of
<Z_0> over a world-size-2 gloo group with the oracle as each rank's executor."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from rustatevec_b200.circuits import ansatz_batch
from rustatevec_b200.shard import circuit_cost, execute_batch_sharded, lpt_partition


def test_lpt_partition_covers_every_index_once_and_balances():
    rng = np.random.default_rng(0)
    costs = list(rng.integers(1, 1000, size=101).astype(float))
    for world in (1, 2, 3, 8):
        parts = lpt_partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: max load <= mean load + largest item
        assert max(loads) <= sum(costs) / world + max(costs)
    assert lpt_partition([], 2) == [[], []]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_cost_model_orders_by_amplitude_work():
    cs = ansatz_batch(4, 3, n_lo=10, n_hi=12, d_lo=2, d_hi=2)
    for c in cs:
        assert circuit_cost(c) == float(1 << c.n_qubits()) * len(c)


def _oracle_share(circuits):
    z0, probs = [], []
    for c in circuits:
        re, im = oracle.run(c, oracle.REF, oracle.F64)
        p = re * re + im * im
        z0.append(oracle.expectation_z(p, 1))
        probs.append(p)
    return z0, probs


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        circuits = ansatz_batch(9, 5, n_lo=3, n_hi=9, d_lo=1, d_hi=4)
        z_all, mine, probs = execute_batch_sharded(_oracle_share, circuits, world, rank)
        out[rank] = (z_all, mine, len(probs))
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_matches_single_process():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    circuits = ansatz_batch(9, 5, n_lo=3, n_hi=9, d_lo=1, d_hi=4)
    want, _ = _oracle_share(circuits)
    z0_r0, mine0, n0 = out[0]
    z0_r1, mine1, n1 = out[1]
    assert z0_r0 == z0_r1
    assert np.allclose(z0_r0, want, atol=0, rtol=0)
    assert sorted(mine0 + mine1) == list(range(9)) and n0 == len(mine0) and n1 == len(mine1)
