"""The benchmark configurations at full size, checked by size-independent properties where no host
oracle can hold the state, and against the oracle where it can:

* QFT(32) complex64 on an i.i.d. complex Gaussian input: 1-F of the learned plan against a
  complex128 run of the same circuit on the same input <= 1e-5 (crates/qsv-core/src/circuits.rs:61-74);
* QAOA MaxCut 33 qubits complex128 (a 137 GB state): FP64 norm = 1 to 1e-14, and the learned plan
  equals the greedy plan to 1e-12 on <Z> for five masks and on a set of amplitudes;
* the batched configuration, 4096 uneven ansatz circuits in both precisions: <Z_0> of every
  circuit against its complex128 twin, and a seeded 512-circuit subset's probabilities and <Z_0>
  against the oracle's CpuBackend restatement per circuit (crates/qsv-core/src/sample.rs:177-200).
"""
import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend, Plan, PLAN_GREEDY, PLAN_LEARNED, ENGINE_AUTO, ENGINE_CUDA_CORE
from rustatevec_b200 import _lib as L
from rustatevec_b200 import tuning
from rustatevec_b200.circuits import ansatz_batch, qaoa_maxcut, qft

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def trained_model(built):
    tuning.load()
    yield
    tuning.install(None)


def test_qft32_learned_plan_fidelity_vs_complex128(built):
    n, seed = 32, 0
    circ = qft(n)
    be = B200Backend(0, precision="f32")
    be64 = B200Backend(0, precision="f64")
    try:
        st = be.alloc(n)                     # 32 GiB
        be.init_gaussian(st, seed)
        p = Plan(be, circ, L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO))
        p.run(st)
        s64 = be64.alloc(n)                  # 64 GiB
        be64.init_gaussian(s64, seed)
        be64.run(s64, circ, L.make_opts(L.PLAN_TILE, 4, ENGINE_AUTO))
        ip = be.inner_product(st, s64)
        inf = 1.0 - abs(ip) ** 2 / (be.norm_sqr(st) * be64.norm_sqr(s64))
        assert inf <= 1e-5, inf
        assert abs(be64.norm_sqr(s64) - 1.0) < 1e-12
        p.free()
        s64.free()
        st.free()
    finally:
        be64.close()
        be.close()


def test_qaoa33_c128_invariants_and_learned_equals_greedy(built):
    n = 33
    circ = qaoa_maxcut(n, 4, 0)
    be = B200Backend(0, precision="f64")
    try:
        st = be.alloc(n)                     # 128 GiB: one state at a time
        masks = [1, 3, 1 << (n - 1), (1 << n) - 1, 0x5555555555555555 & ((1 << n) - 1)]
        idx = [0, 12345, (1 << n) - 1, 0xABCDEF01, 1 << 32]
        out = {}
        for name, opts in (("learned", L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO)),
                           ("greedy", L.make_opts(PLAN_GREEDY, 4, ENGINE_CUDA_CORE))):
            p = Plan(be, circ, opts)
            be.init_basis(st, 0)
            p.run(st)
            out[name] = {"norm": be.norm_sqr(st), "z": [be.expectation_z(st, m) for m in masks],
                         "amp": [be.amplitude(st, i) for i in idx]}
            p.free()
        for name, v in out.items():
            assert abs(v["norm"] - 1.0) <= 1e-14, (name, v["norm"] - 1.0)
        dz = max(abs(a - b) for a, b in zip(out["learned"]["z"], out["greedy"]["z"]))
        da = max(abs(a - b) for a, b in zip(out["learned"]["amp"], out["greedy"]["amp"]))
        assert dz <= 1e-12 and da <= 1e-12, (dz, da)
        st.free()
    finally:
        be.close()


def test_batched_4096_ansatz_circuits_both_precisions(built):
    circuits = ansatz_batch(4096, 0)
    res = {}
    for prec in ("f32", "f64"):
        be = B200Backend(0, precision=prec)
        try:
            z0, probs, st = be.execute_batch(circuits)
            res[prec] = (z0, probs)
        finally:
            be.close()
    z32, p32 = res["f32"]
    z64, p64 = res["f64"]
    assert np.max(np.abs(z32 - z64)) <= 2e-5
    rng = np.random.default_rng(4096)
    subset = rng.choice(len(circuits), size=512, replace=False)
    for i in subset:
        c = circuits[int(i)]
        re, im = oracle.run(c, oracle.CPU_PARALLEL, oracle.F64)
        want = re * re + im * im
        zw = oracle.expectation_z(want, 1)
        assert np.max(np.abs(p64[int(i)] - want)) <= 2e-12, int(i)
        assert np.max(np.abs(p32[int(i)] - want)) <= 2e-5, int(i)
        assert abs(z64[int(i)] - zw) <= 2e-12, int(i)
        assert abs(z32[int(i)] - zw) <= 2e-5, int(i)
