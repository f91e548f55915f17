"""The batched persistent runner (qsvb_execute_batch): every circuit of a batch against the
oracle (RefBackend restatement run per circuit, then expectation_z(probs, 1) as in
crates/qsv-core/src/sample.rs:177-200), for whole-in-shared-memory circuits and for circuits that
take several passes over HBM, in both precisions."""
import ctypes as C

import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend, DenseGate
from rustatevec_b200 import _lib as L
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import SplitMix64, ansatz_batch, ansatz_circuit, random_circuit

pytestmark = pytest.mark.gpu

# probabilities are |amp|^2 <= 1: the amplitude tolerance carries over (x2 for the square)
TOL = {"f64": 2e-12, "f32": 2e-5}


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def oracle_probs(c):
    re, im = oracle.run(c, oracle.REF, oracle.F64)
    return re * re + im * im


def check_batch(be, circuits, local_qubits=0, register_qubits=0):
    pb = L.PackedBatch(circuits)
    z0 = np.zeros(len(circuits))
    sizes = [1 << c.n_qubits() for c in circuits]
    probs = np.zeros(sum(sizes))
    st = L.PlanStats()
    L.check(L.lib().qsvb_execute_batch_ex(be.ctx, pb.ptr(), len(circuits), be.dtype, local_qubits,
                                          register_qubits, z0.ctypes.data_as(C.POINTER(C.c_double)),
                                          probs.ctypes.data_as(C.POINTER(C.c_double)), None, C.byref(st)))
    off = 0
    for i, c in enumerate(circuits):
        want = oracle_probs(c)
        got = probs[off:off + sizes[i]]
        off += sizes[i]
        assert np.max(np.abs(got - want)) <= TOL[be.precision], (i, c.n_qubits(), local_qubits)
        zerr = abs(z0[i] - oracle.expectation_z(want, 1))
        assert zerr <= TOL[be.precision], (i, zerr)
    return st.to_dict()


def test_ansatz_batch_whole_circuits_in_shared_memory(be):
    circuits = ansatz_batch(64, 11, n_lo=2, n_hi=13, d_lo=1, d_hi=6)
    st = check_batch(be, circuits)
    assert st["n_sweeps"] == 64  # one pass per circuit


def register_widths(be):
    return (3, 4) if be.precision == "f64" else (4, 5)


@pytest.mark.parametrize("local_qubits", [7, 9, 12])
@pytest.mark.parametrize("narrow", [False, True])
def test_multi_pass_circuits(be, local_qubits, narrow):
    rng = SplitMix64(local_qubits)
    circuits = [ansatz_circuit(n, 3 + n % 4, rng) for n in (8, 11, 13, 16)]
    circuits += [random_circuit(n, 30 * n, 100 + n) for n in (9, 12, 15, 17)]
    st = check_batch(be, circuits, local_qubits, register_widths(be)[0 if narrow else 1])
    assert st["n_sweeps"] > len(circuits)


def test_uneven_mix_default_tiles(be):
    rng = SplitMix64(5)
    circuits = [ansatz_circuit(n, d, rng) for n, d in ((18, 5), (3, 12), (14, 9), (16, 4), (2, 1), (15, 7))]
    circuits += [random_circuit(n, 200, n) for n in (4, 10, 17)]
    for rq in register_widths(be):
        check_batch(be, circuits, 0, rq)


def test_generic_two_qubit_gates_any_order(be):
    c = Circuit(12)
    for q in range(12):
        c.h(q)
    for a, b in ((11, 0), (3, 9), (0, 11), (7, 2), (5, 6), (10, 1)):
        c.rzz(a, b, 0.3 + a).cx(a, b).swap(b, a).cz(a, b)
    for rq in register_widths(be):
        check_batch(be, [c], 7, rq)
        check_batch(be, [c], 0, rq)


def test_empty_circuits_and_probability_offsets(be):
    circuits = [Circuit(3), Circuit(9), Circuit(1)]
    circuits[1].x(4)
    pb = L.PackedBatch(circuits)
    offsets = np.array([600, 0, 700], dtype=np.uint64)
    probs = np.full(800, -1.0)
    z0 = np.zeros(3)
    L.check(L.lib().qsvb_execute_batch(be.ctx, pb.ptr(), 3, be.dtype, z0.ctypes.data_as(C.POINTER(C.c_double)),
                                       probs.ctypes.data_as(C.POINTER(C.c_double)),
                                       offsets.ctypes.data_as(C.POINTER(C.c_uint64)), None))
    assert probs[600] == 1.0 and np.all(probs[601:608] == 0)
    assert probs[16] == 1.0 and np.sum(probs[:512]) == 1.0
    assert probs[700] == 1.0 and probs[701] == 0.0
    assert np.all(probs[512:600] == -1.0) and np.all(probs[702:] == -1.0)
    assert list(z0) == [1.0, 1.0, 1.0]


def test_reusable_batch_object_and_autotune(be):
    circuits = ansatz_batch(24, 9, n_lo=8, n_hi=17, d_lo=2, d_hi=8)
    pb = L.PackedBatch(circuits)
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.qsvb_batch_create(be.ctx, pb.ptr(), pb.count, be.dtype, 0, 0, C.byref(h)))
    try:
        runs = []
        for _ in range(3):  # graph replays: same results every time
            z0 = np.zeros(pb.count)
            L.check(lib.qsvb_batch_run(be.ctx, h, z0.ctypes.data_as(C.POINTER(C.c_double)), None, None, None))
            runs.append(z0)
        assert np.array_equal(runs[0], runs[1]) and np.array_equal(runs[0], runs[2])
        for i, c in enumerate(circuits):
            assert abs(runs[0][i] - oracle.expectation_z(oracle_probs(c), 1)) <= 1e-4
    finally:
        L.check(lib.qsvb_batch_free(be.ctx, h))
    best_l, best_r = C.c_uint32(), C.c_uint32()
    secs = np.zeros(8)
    count = C.c_size_t()
    L.check(lib.qsvb_batch_autotune(be.ctx, pb.ptr(), pb.count, be.dtype, C.byref(best_l), C.byref(best_r),
                                    secs.ctypes.data_as(C.POINTER(C.c_double)), 8, C.byref(count)))
    top = 13 if be.precision == "f64" else 14
    assert top - 2 <= best_l.value <= top and best_r.value in register_widths(be)
    assert count.value == 6 and np.all(secs[:6] > 0)
    assert np.min(secs[:6]) == secs[2 * (best_l.value - (top - 2)) + register_widths(be).index(best_r.value)]


def test_planning_on_several_host_threads_gives_the_same_batch(be, monkeypatch):
    """Circuits are planned in chunks on host threads and concatenated; the device results are
    bit-identical whatever the number of chunks."""
    rng = SplitMix64(77)
    circuits = ansatz_batch(40, 9, n_lo=2, n_hi=12, d_lo=1, d_hi=5)
    circuits += [ansatz_circuit(n, 4, rng) for n in (13, 15, 17)] + [random_circuit(n, 25 * n, n) for n in (14, 16)]
    rng2 = np.random.default_rng(0)
    order = rng2.permutation(len(circuits))
    circuits = [circuits[i] for i in order]
    out = []
    for threads in ("1", "3", "7", "64"):
        monkeypatch.setenv("QSVB_BATCH_PLAN_THREADS", threads)
        z0, probs, st = be.execute_batch(circuits, local_qubits=10)
        out.append((z0, np.concatenate(probs), st["n_sweeps"], st["algorithmic_bytes"]))
    for z0, p, n, b in out[1:]:
        assert np.array_equal(z0, out[0][0]) and np.array_equal(p, out[0][1])
        assert n == out[0][2] and b == pytest.approx(out[0][3], rel=1e-12)
    monkeypatch.delenv("QSVB_BATCH_PLAN_THREADS")
    check_batch(be, circuits, 10)


def test_backend_execute_batch_matches_single_circuit_path(be):
    circuits = ansatz_batch(6, 3, n_lo=10, n_hi=16, d_lo=2, d_hi=4)
    z0, probs, st = be.execute_batch(circuits)
    for i, c in enumerate(circuits):
        s = be.execute(c)
        p = be.probabilities(s, fp64=True)
        assert np.max(np.abs(probs[i] - p)) <= TOL[be.precision]
        assert abs(z0[i] - be.expectation_z(s, 1)) <= (1e-4 if be.precision == "f32" else 1e-10)
        s.free()
    assert st["measured_seconds"] > 0 and st["predicted_seconds"] == 0


def test_batch_rejects_invalid_input(be):
    three = Circuit(4)
    three.push(DenseGate(3, np.eye(8, dtype=complex)), [0, 1, 2])
    cases = (([three], 0, 0), ([Circuit(31)], 0, 0), ([Circuit(4)], 15, 0), ([Circuit(4)], 5, 0),
             ([Circuit(4)], 0, 2), ([Circuit(4)], 0, 6))
    for circuits, lq, rq in cases:
        pb = L.PackedBatch(circuits)
        z0 = np.zeros(1)
        rc = L.lib().qsvb_execute_batch_ex(be.ctx, pb.ptr(), 1, be.dtype, lq, rq,
                                           z0.ctypes.data_as(C.POINTER(C.c_double)), None, None, None)
        assert rc == L.QSVB_E_INVALID, (circuits[0].n_qubits(), lq, rq)
    assert L.lib().qsvb_execute_batch(be.ctx, None, 0, be.dtype, None, None, None, None) == L.QSVB_E_INVALID


def test_dependency_wait_that_runs_out_fails_the_run_and_the_context_recovers(be):
    """A multi-pass batch with a dependency-wait budget of one clock64 cycle: the tiles of pass 1
    that are taken while pass 0 is still running give up at once, the run returns QSVB_E_TIMEOUT,
    and with the default budget restored the same batch object runs correctly on the same context."""
    rng = SplitMix64(2024)
    circuits = [ansatz_circuit(20, 6, rng), ansatz_circuit(19, 5, rng)]
    pb = L.PackedBatch(circuits)
    lib = L.lib()
    h = C.c_void_p()
    L.check(lib.qsvb_batch_create(be.ctx, pb.ptr(), pb.count, be.dtype, 12, 0, C.byref(h)))
    try:
        z0 = np.zeros(pb.count)
        zp = z0.ctypes.data_as(C.POINTER(C.c_double))
        st = L.PlanStats()
        L.check(lib.qsvb_batch_run(be.ctx, h, zp, None, None, C.byref(st)))
        assert st.n_sweeps >= 4  # several passes over HBM per circuit: tiles wait on earlier passes
        L.check(lib.qsvb_batch_set_wait_budget(be.ctx, h, 1))
        codes = [lib.qsvb_batch_run(be.ctx, h, zp, None, None, None) for _ in range(3)]
        assert L.QSVB_E_TIMEOUT in codes, codes
        assert "budget" in lib.qsvb_last_error().decode()
        L.check(lib.qsvb_batch_set_wait_budget(be.ctx, h, 0))
        L.check(lib.qsvb_batch_run(be.ctx, h, zp, None, None, None))
        for i, c in enumerate(circuits):
            want = oracle.expectation_z(oracle_probs(c), 1)
            assert abs(z0[i] - want) <= TOL[be.precision], (i, z0[i], want)
        assert lib.qsvb_batch_set_wait_budget(be.ctx, h, 1 << 41) == L.QSVB_E_INVALID
    finally:
        L.check(lib.qsvb_batch_free(be.ctx, h))
