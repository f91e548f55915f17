"""A state spread over 2^g slices on one B200 (every rank in this process): the CUDA engine runs
each slice's local steps and blocks swap by device copies on the engine's stream. Checked against
the oracle's run of the whole circuit (complex128 max |d amp| <= 1e-12, complex64 <= 1e-5) and
against the single-state engine at a larger size."""
import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend
from rustatevec_b200.circuit import Circuit
from rustatevec_b200 import gate as G
from rustatevec_b200.circuits import brickwork, ghz_chain, qaoa_maxcut, qft, random_circuit
from rustatevec_b200.distributed import B200SliceEngine, DistributedState, TorchComm

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def circuits(n):
    c = Circuit(n)
    for q in range(n):
        c.h(q)
    c.cx(n - 1, 0).cz(n - 2, n - 1).cphase(n - 1, 1, 0.3).rzz(n - 3, n - 1, 0.7)
    c.push(G.controlled_1q(G.ry(0.4)), [n - 1, n - 2])
    c.swap(0, n - 1)
    return [random_circuit(n, 10 * n, 5 + n), qft(n), brickwork(n, 4, n), ghz_chain(n), qaoa_maxcut(n, 2, n), c]


@pytest.mark.parametrize("g", [1, 2, 3])
def test_slices_match_the_oracle(be, g):
    n = 13
    eng = B200SliceEngine(be)
    for c in circuits(n):
        ds = DistributedState(n, g, eng, chunk_elems=1000)
        ds.init_basis(0)
        ds.run(c)
        re, im = oracle.run(c, oracle.REF, oracle.F64)
        want = re + 1j * im
        assert np.max(np.abs(ds.gather() - want)) < TOL[be.precision]
        p = np.abs(want) ** 2
        for mask in (0, 1, 1 << (n - 1), (1 << n) - 1):
            assert abs(ds.expectation_z(mask) - oracle.expectation_z(p, mask)) < TOL[be.precision]
        ds.free()


def test_matches_the_single_state_engine(be):
    n, g = 22, 2
    c = random_circuit(n, 300, 77)
    st = be.alloc(n)
    be.init_basis(st, 0)
    be.run(st, c)
    want = be.download(st).as_complex()
    st.free()
    ds = DistributedState(n, g, B200SliceEngine(be))
    ds.init_basis(0)
    stats = ds.run(c)
    assert stats["exchanges"] > 0
    got = ds.gather()
    assert abs(np.vdot(want, got)) ** 2 > 1 - TOL[be.precision]
    assert abs(ds.norm_sqr() - 1) < TOL[be.precision]
    ds.free()


def test_nccl_communicator_on_one_rank(be):
    """TorchComm over a one-rank NCCL group (reductions and the gather run through NCCL on the
    device); the block exchange itself needs two GPUs and is covered by the gloo tests."""
    import datetime
    import socket
    import torch.distributed as dist
    if dist.is_initialized():
        pytest.skip("a process group already exists")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        comm = TorchComm()
        assert comm.device.type == "cuda" and comm.size == 1
        n = 12
        c = random_circuit(n, 80, 4)
        ds = DistributedState(n, 0, B200SliceEngine(be), comm)
        ds.init_basis(0)
        ds.run(c)
        re, im = oracle.run(c, oracle.REF, oracle.F64)
        want = re + 1j * im
        assert np.max(np.abs(ds.gather() - want)) < TOL[be.precision]
        p = np.abs(want) ** 2
        assert abs(ds.expectation_z(0b101) - oracle.expectation_z(p, 0b101)) < TOL[be.precision]
        ds.free()
    finally:
        dist.destroy_process_group()
