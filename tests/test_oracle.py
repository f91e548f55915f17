"""The oracle pinned against the reference's own known answers, and cross-checked three ways:
RefBackend restatement vs CpuBackend restatement vs an independent numpy contraction.
Mirrors crates/qsv-core/tests/{oracle,equivalence,sampling}.rs and the inline unit tests."""
import math

import numpy as np
import pytest

import oracle
from rustatevec_b200 import gate as G
from rustatevec_b200.circuit import Circuit
from rustatevec_b200.circuits import SplitMix64, ghz, qft, random_circuit

from helpers import circuit_from_spec, known_answers, max_abs_diff, numpy_run

KA = known_answers()
TOL = 1e-9  # crates/qsv-core/tests/equivalence.rs:26


def cplx(re_im):
    return re_im[0] + 1j * re_im[1]


@pytest.mark.parametrize("name", sorted(KA["circuits"]))
@pytest.mark.parametrize("engine", [oracle.REF, oracle.CPU_SERIAL, oracle.CPU_PARALLEL])
def test_known_answer_circuits(name, engine):
    spec = KA["circuits"][name]
    c = circuit_from_spec(spec["n"], spec["ops"])
    re, im = oracle.run(c, engine, oracle.F64)
    psi = re + 1j * im
    for idx, want in spec["amps"].items():
        assert abs(psi[int(idx)] - cplx(want)) < spec["tol"], (name, idx)
    if "norm" in spec:
        assert abs(oracle.norm_sqr(re, im) - spec["norm"]) < spec["tol"]
    if "others_abs2_below" in spec:
        for i in range(1, len(psi) - 1):
            assert abs(psi[i]) ** 2 < spec["others_abs2_below"]


def test_random_circuits_three_oracles():
    # equivalence.rs:28-70: 200 seeds, n = 3..8, depth 20..59
    for seed in range(200):
        n = 3 + seed % 6
        c = random_circuit(n, 20 + seed % 40, seed)
        ref = oracle.run(c, oracle.REF)
        cpu = oracle.run(c, oracle.CPU_SERIAL)
        par = oracle.run(c, oracle.CPU_PARALLEL)
        a = ref[0] + 1j * ref[1]
        assert max_abs_diff(a, cpu[0] + 1j * cpu[1]) < TOL, seed
        assert max_abs_diff(a, par[0] + 1j * par[1]) < TOL, seed
        assert max_abs_diff(a, numpy_run(c)) < TOL, seed
        assert abs(oracle.norm_sqr(*cpu) - 1.0) < 1e-8


def test_ten_and_fourteen_qubit_suites():
    # equivalence.rs:72-106
    for seed in range(15):
        c = random_circuit(10, 80, 9000 + seed)
        a, b = oracle.run(c, oracle.REF), oracle.run(c, oracle.CPU_SERIAL)
        assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL
    for seed in range(6):
        c = random_circuit(14, 60, 4242 + seed)
        a, b = oracle.run(c, oracle.REF), oracle.run(c, oracle.CPU_PARALLEL)
        assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL


def test_f32_engines_agree_with_f64():
    for seed in range(20):
        c = random_circuit(6, 40, 100 + seed)
        a = oracle.run(c, oracle.REF, oracle.F64)
        b = oracle.run(c, oracle.CPU_SERIAL, oracle.F32)
        assert max_abs_diff(a[0] + 1j * a[1], b[0].astype(np.float64) + 1j * b[1]) < 1e-5


def test_qft_uniform_and_vs_oracle():
    spec = KA["qft_uniform"]
    for n in spec["ns"]:
        re, im = oracle.run(qft(n), oracle.CPU_SERIAL)
        assert np.all(np.abs(re * re + im * im - 2.0 ** -n) < spec["tol"])
    for n in (2, 3, 5, 8):  # equivalence.rs:122-134
        a, b = oracle.run(qft(n), oracle.REF), oracle.run(qft(n), oracle.CPU_PARALLEL)
        assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL


def test_fusion_preserves_results():
    # equivalence.rs:148-178
    for mq in (2, 3, 4, 5):
        for seed in range(40):
            n = 4 + seed % 5
            c = random_circuit(n, 50, 70000 + seed)
            fa, fq, fm = oracle.fuse(c, mq)
            assert len(fa) <= len(c)
            fused = Circuit.from_flat(n, fa, fq, fm)
            a = oracle.run(c, oracle.REF)
            b = oracle.run(fused, oracle.CPU_PARALLEL)
            assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL, (mq, seed)
    for n in (4, 6, 8):
        c = qft(n)
        fused = Circuit.from_flat(n, *oracle.fuse(c, 4))
        a, b = oracle.run(c, oracle.REF), oracle.run(fused, oracle.CPU_PARALLEL)
        assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL


def test_fusion_counts():
    # fusion.rs:162-185
    c = qft(6)
    assert len(oracle.fuse(c, 4)[0]) < len(c)
    d = Circuit(4)
    d.h(0).h(2)
    assert len(oracle.fuse(d, 1)[0]) == 2


def ccx():
    m = np.zeros((8, 8), dtype=np.complex128)
    for i in range(8):
        m[i, {3: 7, 7: 3}.get(i, i)] = 1.0
    return G.DenseGate(3, m)


def test_toffoli_orderings():
    # equivalence.rs:180-225
    for seed, qs in [(1, [0, 1, 2]), (2, [2, 0, 4]), (3, [4, 3, 1]), (4, [5, 2, 0])]:
        c = random_circuit(6, 40, seed)
        c.push(ccx(), qs)
        c.h(0).rx(3, 0.9)
        c.push(ccx(), [1, 4, 5])
        a, b = oracle.run(c, oracle.REF), oracle.run(c, oracle.CPU_SERIAL)
        assert max_abs_diff(a[0] + 1j * a[1], b[0] + 1j * b[1]) < TOL
        assert max_abs_diff(a[0] + 1j * a[1], numpy_run(c)) < TOL


def test_expectation_z():
    spec = KA["expz_ghz5"]
    re, im = oracle.run(ghz(spec["n"]), oracle.CPU_PARALLEL)
    p = oracle.probabilities(re, im)
    for mask, want in zip(spec["masks"], spec["values"]):
        assert abs(oracle.expectation_z(p, mask) - want) < spec["tol"]
    for probs, mask, want in KA["expz_basic"]["cases"]:
        assert abs(oracle.expectation_z(np.array(probs), mask) - want) < 1e-12


def test_gate_library_matches_oracle_and_reference_unit_tests():
    for name, fn in G.LIBRARY.items():
        th = 0.7321 if name in G.PARAMETRIC else None
        ours = fn(th).matrix if th is not None else fn().matrix
        theirs = oracle.gate(name, th or 0.0)
        assert np.array_equal(ours, theirs), name
    # gate.rs:193-205 CX permutation
    cxm = G.cx().matrix
    for col, row in enumerate(KA["cx_permutation"]["col_to_row"]):
        for r in range(4):
            assert cxm[r, col] == (1.0 if r == row else 0.0)
    # gate.rs:223-239 is_diagonal classes
    for name, th in KA["is_diagonal"]["diagonal"]:
        assert oracle.is_diagonal(oracle.gate(name, th)) and (G.LIBRARY[name](th) if name in G.PARAMETRIC else G.LIBRARY[name]()).is_diagonal()
    for name, th in KA["is_diagonal"]["dense"]:
        assert not oracle.is_diagonal(oracle.gate(name, th))
    # gate.rs:241-247 RZ unit modulus
    rz = G.rz(0.7).matrix
    assert abs(abs(rz[0, 0]) - 1) < 1e-12 and abs(abs(rz[1, 1]) - 1) < 1e-12 and rz[0, 1] == 0


def test_layout_helpers():
    L = oracle.lib()
    for i in range(32):
        assert L.orc_insert_zero_bit(i, 0) == i << 1
    for i, b, want in KA["layout"]["insert_zero_bit"]:
        assert L.orc_insert_zero_bit(i, b) == want
    for i in range(64):
        for b in range(6):
            assert (L.orc_insert_zero_bit(i, b) >> b) & 1 == 0
    for bit in range(5):
        for i in range(16):
            a0 = L.orc_insert_zero_bit(i, bit)
            assert (a0 ^ (a0 | (1 << bit))) == 1 << bit
    for idx, qs, want in KA["layout"]["gather_bits"]:
        q = np.array(qs, np.uint32)
        assert L.orc_gather_bits(idx, q, len(q)) == want
        for sub in range(8):
            assert L.orc_gather_bits(L.orc_scatter_bits(sub, q, 3), q, 3) == sub
    t = np.array(KA["layout"]["tiles"]["targets"], np.uint32)
    seen = set()
    for o in range(4):
        base = L.orc_insert_zero_bits(o, t, 2)
        for s in range(4):
            full = base | L.orc_scatter_bits(s, t, 2)
            assert full not in seen
            seen.add(full)
    assert seen == set(range(16))


def test_complex_mul_and_rng():
    a, b = KA["complex_mul"]["a"], KA["complex_mul"]["b"]
    assert cplx(a) * cplx(b) == cplx(KA["complex_mul"]["ab"])
    # circuits.rs:115-128: determinism and unit() range; product RNG == oracle RNG stream
    import ctypes
    r1, r2 = SplitMix64(42), SplitMix64(42)
    st = ctypes.c_uint64(42)
    for _ in range(100):
        v = r1.next_u64()
        assert v == r2.next_u64() == oracle.lib().orc_splitmix_next(ctypes.byref(st))
    r = SplitMix64(1)
    for _ in range(1000):
        assert 0.0 <= r.unit() < 1.0
    # published SplitMix64 test value (seed 0, first output)
    assert SplitMix64(0).next_u64() == 0xE220A8397B1DCDAF


def test_generators_shape():
    # circuits.rs:130-138
    assert len(ghz(5)) == 5
    assert qft(4).n_qubits() == 4
    assert len(random_circuit(4, 30, 7)) == 30


def test_circuit_push_validation():
    # circuit.rs:54-78 panics -> ValueError
    c = Circuit(3)
    with pytest.raises(ValueError):
        c.push(G.cx(), [0])
    with pytest.raises(ValueError):
        c.push(G.h(), [3])
    with pytest.raises(ValueError):
        c.push(G.cx(), [1, 1])


def test_samplers_against_the_reference_unit_tests():
    """Host samplers: the alias table (sample.rs:217-232) and the cdf_sample restatement
    (sample.rs:163-172), on the reference's own test distributions and SplitMix64 seeds."""
    from rustatevec_b200.circuits import SplitMix64
    from rustatevec_b200.sample import alias_sample
    w = np.array([0.1, 0.6, 0.0, 0.3])
    counts = np.bincount(alias_sample(w, 40000, SplitMix64(0xDEADBEEF)), minlength=4)
    assert counts[2] == 0
    assert np.max(np.abs(counts / 40000 - w)) < 0.01
    idx, u, cdf = oracle.cdf_sample(w, 40000, 0xDEADBEEF)
    assert np.count_nonzero(idx == 2) == 0 and np.max(np.abs(np.bincount(idx, minlength=4) / 40000 - w)) < 0.01
    # the vectorised stream equals the scalar generator, and the rule is a lower bound
    r = SplitMix64(5)
    assert np.array_equal(oracle.splitmix_units(5, 16), np.array([r.unit() for _ in range(16)]))
    cdf = np.cumsum([0.0, 0.5, 0.5])
    assert int(np.searchsorted(cdf, 0.5, side="left")) == 1  # u on a boundary takes the lower outcome
    w2 = np.array([0.25, 0.25, 0.4, 0.1])
    a = np.bincount(alias_sample(w2, 40000, SplitMix64(1)), minlength=4) / 40000
    b = np.bincount(oracle.cdf_sample(w2, 40000, 2)[0], minlength=4) / 40000
    assert np.max(np.abs(a - b)) < 0.02
