"""GPU parity: the CUDA engine through the C ABI vs the oracle (RefBackend / CpuBackend
restatements) on the same circuits and seeds. Mirrors crates/qsv-cuda/tests/equivalence.rs and
the core differential suite, with the tolerances stated per precision:
complex128 max |d amp| <= 1e-12, complex64 max |d amp| <= 1e-5."""
import math

import numpy as np
import pytest

import oracle
from rustatevec_b200 import (B200Backend, FusionConfig, PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_LEARNED,
                             PLAN_WINDOW, ENGINE_CUDA_CORE, QsvbError, fuse)
from rustatevec_b200 import _lib as L
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import ghz, ghz_chain, qft, random_circuit

from helpers import circuit_from_spec, infidelity, known_answers, max_abs_diff

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


def ref_state(c, psi0=None):
    if psi0 is None:
        re, im = oracle.run(c, oracle.REF, oracle.F64)
    else:
        re, im = oracle.run(c, oracle.REF, oracle.F64, state=(psi0.real.copy(), psi0.imag.copy()))
    return re + 1j * im


def gpu_state(be, c, psi0=None, opts=None):
    st = be.alloc(c.n_qubits())
    if psi0 is None:
        be.init_basis(st, 0)
    else:
        be.upload(st, psi0.real, psi0.imag)
    be.run(st, c, opts)
    return be.download(st).as_complex()


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def haar(k, seed):
    rng = np.random.default_rng(seed)
    z = (rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))) / math.sqrt(2)
    q, r = np.linalg.qr(z)
    return q * (np.diag(r) / np.abs(np.diag(r)))


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def opts(planner=PLAN_AS_GIVEN, k=4, engine=0, graph=True):
    return L.make_opts(planner, k, engine, graph)


# --------------------------------------------------------------- crates/qsv-cuda/tests/equivalence.rs
def test_cuda_matches_oracle_on_random_circuits(be):
    for seed in range(40):
        n = 3 + seed % 6
        c = random_circuit(n, 20 + seed % 40, 0xABCD0000 ^ seed)
        want = ref_state(c)
        got = be.download(be.execute(c)).as_complex()
        assert max_abs_diff(want, got) < TOL[be.precision], (seed, n)


def test_cuda_matches_oracle_qft_and_ghz(be):
    for n in (2, 3, 5, 8):
        assert max_abs_diff(ref_state(qft(n)), be.download(be.execute(qft(n))).as_complex()) < TOL[be.precision]
    for n in (3, 6, 10):
        assert max_abs_diff(ref_state(ghz(n)), be.download(be.execute(ghz(n))).as_complex()) < TOL[be.precision]


def test_cuda_probabilities_sum_to_one(be):
    st = be.execute(qft(10))
    p = be.probabilities(st)
    assert abs(float(np.sum(p, dtype=np.float64)) - 1.0) < (1e-12 if be.precision == "f64" else 1e-6)
    assert abs(be.norm_sqr(st) - 1.0) < (1e-12 if be.precision == "f64" else 1e-6)


# --------------------------------------------------------------- core differential suite on the GPU
def test_known_answers_on_gpu(be):
    ka = known_answers()["circuits"]
    for name, spec in ka.items():
        c = circuit_from_spec(spec["n"], spec["ops"])
        got = be.download(be.execute(c)).as_complex()
        tol = max(spec["tol"], TOL[be.precision])
        for idx, want in spec["amps"].items():
            assert abs(got[int(idx)] - complex(*want)) < tol, (name, idx)


def test_trait_default_loop_of_apply(be):
    # Backend::execute's default body: alloc, init_basis(0), apply per op (mod.rs:66-73)
    for seed in range(30):
        n = 3 + seed % 10
        c = random_circuit(n, 40, 5000 + seed)
        st = be.alloc(n)
        be.init_basis(st, 0)
        for op in c.ops():
            be.apply(st, op.gate, op.qubits)
        assert max_abs_diff(ref_state(c), be.download(st).as_complex()) < TOL[be.precision], seed


@pytest.mark.parametrize("planner", [PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_WINDOW, PLAN_LEARNED])
def test_all_planners_match_unfused_oracle(be, planner):
    for k in (2, 3, 4, 5, 6):
        for seed in range(12):
            n = 4 + seed % 10
            c = random_circuit(n, 60, 70000 + 17 * k + seed)
            got = gpu_state(be, c, opts=opts(planner, k))
            want = ref_state(c)
            err = max_abs_diff(want, got)
            assert err < TOL[be.precision], (planner, k, seed, n, err)
            if be.precision == "f32":
                assert infidelity(want, got) < 1e-5, (planner, k, seed, n)


def test_random_suites_n10_n14(be):
    for seed in range(6):
        c = random_circuit(14, 60, 4242 + seed)
        want, got = ref_state(c), gpu_state(be, c, opts=opts(PLAN_WINDOW, 5))
        err = max_abs_diff(want, got)
        assert err < TOL[be.precision], (seed, err)
        if be.precision == "f32":
            assert infidelity(want, got) < 1e-5, seed
    for seed in range(6):
        c = random_circuit(10, 80, 9000 + seed)
        assert max_abs_diff(ref_state(c), gpu_state(be, c)) < TOL[be.precision]


def test_golden_state_fixtures(be):
    import os
    data = np.load(os.path.join(os.path.dirname(__file__), "golden", "oracle_states.npz"))
    for key in data.files:
        if key.startswith("random_"):
            _, n, d, s = key.split("_")
            c = random_circuit(int(n), int(d), int(s))
        else:
            c = qft(int(key.split("_")[1]))
        got = gpu_state(be, c, opts=opts(PLAN_WINDOW, 4))
        err = max_abs_diff(data[key], got)
        assert err < TOL[be.precision], (key, err)
        if be.precision == "f32":
            assert infidelity(data[key], got) < 1e-5, key


# --------------------------------------------------------------- per-kernel coverage
@pytest.mark.parametrize("n", [5, 12, 14])
def test_one_qubit_every_target(be, n):
    psi = random_state(n, n)
    for t in range(n):
        c = Circuit(n)
        c.push(G.DenseGate(1, haar(1, 100 + t)), [t])
        assert max_abs_diff(ref_state(c, psi), gpu_state(be, c, psi)) < TOL[be.precision], t


@pytest.mark.parametrize("n", [4, 12, 13])
def test_controlled_every_pair(be, n):
    psi = random_state(n, 7 + n)
    u = haar(1, 3)
    cu = G.controlled_1q(G.DenseGate(1, u))
    for ctl in range(n):
        for tgt in range(n):
            if ctl == tgt:
                continue
            c = Circuit(n)
            c.cx(ctl, tgt)
            c.push(cu, [tgt, ctl])
            assert max_abs_diff(ref_state(c, psi), gpu_state(be, c, psi)) < TOL[be.precision], (ctl, tgt)


def ccx():
    m = np.zeros((8, 8), dtype=np.complex128)
    for i in range(8):
        m[i, {3: 7, 7: 3}.get(i, i)] = 1.0
    return G.DenseGate(3, m)


def test_multi_controlled_and_toffoli(be):
    for seed, qs in [(1, [0, 1, 2]), (2, [2, 0, 4]), (3, [4, 3, 1]), (4, [5, 2, 0]), (5, [9, 1, 11]), (6, [3, 10, 0])]:
        c = random_circuit(12, 40, seed)
        c.push(ccx(), qs)
        c.h(0).rx(3, 0.9)
        c.push(ccx(), [1, 4, 5])
        assert max_abs_diff(ref_state(c), gpu_state(be, c)) < TOL[be.precision], seed


@pytest.mark.parametrize("n", [3, 12, 14])
def test_diagonal_gates(be, n):
    psi = random_state(n, 11 * n)
    rng = np.random.default_rng(n)
    for trial in range(20):
        k = 1 + trial % min(n, 6)
        qs = list(rng.choice(n, size=k, replace=False))
        d = np.exp(1j * rng.uniform(0, 2 * math.pi, size=1 << k))
        c = Circuit(n)
        c.push(G.DenseGate(k, np.diag(d)), qs)
        a, b = qs[0], qs[-1] if k > 1 else (qs[0] + 1) % n
        if a != b:
            c.cz(a, b).cphase(b, a, 0.37).rzz(a, b, 1.3)
        assert max_abs_diff(ref_state(c, psi), gpu_state(be, c, psi)) < TOL[be.precision], (trial, qs)


@pytest.mark.parametrize("n", [6, 12, 14])
def test_dense_gates_every_arity(be, n):
    psi = random_state(n, 3 * n)
    rng = np.random.default_rng(1000 + n)
    for k in range(2, 7):
        if k > n:
            continue
        sets = [list(range(k)), list(range(n - k, n)), list(rng.choice(n, size=k, replace=False)),
                list(rng.choice(n, size=k, replace=False))]
        for qs in sets:
            c = Circuit(n)
            c.push(G.DenseGate(k, haar(k, 7 * k + len(qs))), [int(q) for q in qs])
            got = gpu_state(be, c, psi, opts(PLAN_AS_GIVEN, 6, ENGINE_CUDA_CORE))
            err = max_abs_diff(ref_state(c, psi), got)
            assert err < TOL[be.precision], (k, qs, err)


# --------------------------------------------------------------- configs / reductions / errors
def test_ghz24_chain_probabilities_c128(be64):
    c = ghz_chain(24)
    st = be64.execute(c)
    p = be64.probabilities(st)
    re, im = oracle.run(c, oracle.CPU_PARALLEL, oracle.F64)
    want = oracle.probabilities(re, im)
    assert max_abs_diff(p, want) < 1e-12
    assert abs(p[0] - 0.5) < 1e-12 and abs(p[-1] - 0.5) < 1e-12


def test_reductions(be):
    st = be.execute(ghz(5))
    # sampling.rs:49-58 asserts 1e-9 on an f64 state; a complex64 state holds 1/sqrt(2) to 2^-24
    tol = 1e-9 if be.precision == "f64" else 1e-6
    for mask, want in zip([1, 3, 15, 31], [0.0, 1.0, 1.0, 0.0]):
        assert abs(be.expectation_z(st, mask) - want) < tol
    c = random_circuit(12, 80, 77)
    a = be.execute(c)
    want = ref_state(c)
    probs = np.abs(want) ** 2
    for mask in (1, 2, 5, 0x800, 0xFFF):
        sign = np.array([(-1) ** bin(i & mask).count("1") for i in range(len(probs))])
        assert abs(be.expectation_z(a, mask) - float(np.sum(sign * probs))) < (1e-12 if be.precision == "f64" else 1e-5)
    b = be.execute(random_circuit(12, 80, 78))
    wb = ref_state(random_circuit(12, 80, 78))
    ip = be.inner_product(a, b)
    assert abs(ip - np.vdot(want, wb)) < (1e-12 if be.precision == "f64" else 1e-5)
    assert abs(be.fidelity(a, b) - abs(np.vdot(want, wb)) ** 2) < (1e-12 if be.precision == "f64" else 1e-5)
    assert abs(be.amplitude(a, 1234) - want[1234]) < TOL[be.precision]


def host_gaussian(n, seed, dtype):
    G_ = np.uint64(0x9E3779B97F4A7C15)
    i = np.arange(1 << n, dtype=np.uint64)

    def mix(z):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))
    with np.errstate(over="ignore"):
        h1 = mix(np.uint64(seed) + (np.uint64(2) * i + np.uint64(1)) * G_)
        h2 = mix(np.uint64(seed) + (np.uint64(2) * i + np.uint64(2)) * G_)
    u1 = ((h1 >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53
    u2 = (h2 >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    re = (r * np.cos(2 * np.pi * u2)).astype(dtype)
    im = (r * np.sin(2 * np.pi * u2)).astype(dtype)
    nrm = np.sum(re.astype(np.float64) ** 2 + im.astype(np.float64) ** 2)
    return (re / np.sqrt(nrm)).astype(np.float64) + 1j * (im / np.sqrt(nrm)).astype(np.float64)


def test_gaussian_init_matches_host(be):
    st = be.alloc(12)
    be.init_gaussian(st, 0xC0FFEE)
    got = be.download(st).as_complex()
    want = host_gaussian(12, 0xC0FFEE, be.np_real)
    assert max_abs_diff(got, want) < (1e-12 if be.precision == "f64" else 2e-6)
    assert abs(be.norm_sqr(st) - 1.0) < (1e-12 if be.precision == "f64" else 1e-5)


def test_errors_are_status_codes(be):
    st = be.alloc(4)
    with pytest.raises(QsvbError) as e:
        be.init_basis(st, 16)
    assert e.value.code == L.QSVB_E_INVALID
    with pytest.raises(QsvbError) as e:
        be.apply(st, G.h(), [4])
    assert e.value.code == L.QSVB_E_INVALID
    with pytest.raises(QsvbError) as e:
        be.alloc(34 if be.precision == "f64" else 35)
    assert e.value.code in (L.QSVB_E_OOM, L.QSVB_E_INVALID)
    # the context stays usable after every rejected call
    be.init_basis(st, 3)
    assert abs(be.amplitude(st, 3) - 1.0) < 1e-12


# --------------------------------------------------------------- phase-polynomial (QAOA cost layer)
@pytest.mark.parametrize("n", [8, 12, 14])
def test_qaoa_phase_sweeps_match_oracle(be, n):
    from rustatevec_b200.circuits import qaoa_maxcut
    c = qaoa_maxcut(n, 3, 11 + n)
    st = be.alloc(n)
    be.init_basis(st, 0)
    # CUDA-core engine: the phase-polynomial sweep, not a tensor-core chain plan, is under test
    stats = be.run(st, c, opts(PLAN_LEARNED, 4, ENGINE_CUDA_CORE))
    assert stats["by_kind"].get("phase", 0) >= 1, stats
    got = be.download(st).as_complex()
    err = max_abs_diff(ref_state(c), got)
    assert err < TOL[be.precision], (stats, err)


def test_phase_sweep_general_diagonals(be):
    # mixed 1- and 2-qubit diagonal terms, repeated pairs, and a low/high split at bit 12
    n = 14
    rng = np.random.default_rng(5)
    c = Circuit(n)
    for q in range(n):
        c.h(q)
    for _ in range(40):
        a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
        kind = rng.integers(4)
        if kind == 0:
            c.rzz(a, b, float(rng.uniform(0, 6.3)))
        elif kind == 1:
            c.cphase(a, b, float(rng.uniform(0, 6.3)))
        elif kind == 2:
            c.rz(a, float(rng.uniform(0, 6.3)))
        else:
            c.cz(a, b)
    st = be.alloc(n)
    be.init_basis(st, 0)
    stats = be.run(st, c, opts(PLAN_LEARNED, 3))
    got = be.download(st).as_complex()
    err = max_abs_diff(ref_state(c), got)
    assert err < TOL[be.precision], (stats, err)
