"""Device sampling (the backend's ``sample``, qsvb_sample) against the oracle's restatement of
cdf_sample (crates/qsv-core/src/sample.rs:163-172) on the same SplitMix64 stream
(crates/qsv-core/src/circuits.rs:22-46), draw for draw, plus the reference's sampling tests
(crates/qsv-core/tests/sampling.rs: GHZ outcomes, histogram vs probabilities) through the trait
method, and the statistical agreement of the alias and inverse-CDF samplers
(crates/qsv-core/src/sample.rs:234-258)."""
import ctypes as C

import numpy as np
import pytest

import oracle
from rustatevec_b200 import B200Backend
from rustatevec_b200 import _lib as L
from rustatevec_b200.circuits import SplitMix64, ghz, ghz_chain, qft, random_circuit

pytestmark = pytest.mark.gpu

EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def trait_probabilities(be, st):
    """Backend::probabilities as the reference computes it: re*re + im*im in the state's precision."""
    sv = be.download(st)
    re, im = sv.re, sv.im
    return (re * re + im * im).astype(np.float64)


@pytest.mark.parametrize("n", [6, 9, 12, 14, 16, 18])
def test_draw_for_draw_against_cdf_sample(be, n):
    st = be.alloc(n)
    be.init_basis(st, 0)
    be.run(st, random_circuit(n, 10 * n, 40 + n))
    w = trait_probabilities(be, st)
    shots = 20000
    seed = 1234 + n
    got = be.sample_device(st, shots, seed).astype(np.int64)
    want, u, cdf = oracle.cdf_sample(w, shots, seed)
    bad = np.nonzero(got != want)[0]
    # the device's FP64 prefix sums run in another order: a draw may differ only where u lies
    # within rounding of the cumulative value that separates the two outcomes
    tol = 64 * EPS * cdf[-1]
    for k in bad:
        lo, hi = sorted((int(got[k]), int(want[k])))
        gap = np.min(np.abs(cdf[lo:hi] - u[k]))
        assert gap <= tol, (k, int(got[k]), int(want[k]), gap)
    assert len(bad) <= 2, len(bad)
    assert np.all(w[got] > 0)
    st.free()


def test_zero_probability_outcomes_are_never_drawn(be):
    # |psi> with p = [0.1, 0.6, 0, 0.3] (the reference's alias test distribution, sample.rs:217-232)
    w = np.array([0.1, 0.6, 0.0, 0.3])
    st = be.alloc(2)
    be.upload(st, np.sqrt(w), np.zeros(4))
    shots = 200000
    got = be.sample_device(st, shots, 0xDEADBEEF).astype(np.int64)
    want, _, _ = oracle.cdf_sample(trait_probabilities(be, st), shots, 0xDEADBEEF)
    assert np.count_nonzero(got != want) <= 2
    counts = np.bincount(got, minlength=4)
    assert counts[2] == 0
    for k, p in enumerate(w):
        assert abs(counts[k] / shots - p) < 0.01
    st.free()


def test_trait_sample_consumes_the_rng_like_cdf_sample(be):
    st = be.execute(random_circuit(10, 80, 5))
    rng = SplitMix64(99)
    a = be.sample(st, 1000, rng)
    b = be.sample(st, 1000, rng)
    ref = SplitMix64(99)
    for _ in range(2000):
        ref.next_u64()
    assert rng.state == ref.state  # one unit() per shot
    w = trait_probabilities(be, st)
    want_a, _, _ = oracle.cdf_sample(w, 1000, 99)
    want_b, _, _ = oracle.cdf_sample(w, 1000, (99 + 1000 * 0x9E3779B97F4A7C15) & (2 ** 64 - 1))
    assert np.count_nonzero(np.asarray(a) != want_a) + np.count_nonzero(np.asarray(b) != want_b) <= 2


def test_sample_ghz_yields_only_all_zero_or_all_one(be):
    # crates/qsv-core/tests/sampling.rs:8-29 through the trait method
    st = be.execute(ghz(6))
    out = np.asarray(be.sample(st, 50000, SplitMix64(42)))
    assert set(np.unique(out).tolist()) <= {0, 0b111111}
    assert abs(np.count_nonzero(out == 0) / 50000 - 0.5) < 0.02


def test_sample_histogram_matches_probabilities(be):
    # crates/qsv-core/tests/sampling.rs:31-46
    st = be.execute(qft(6))
    p = be.probabilities(st, fp64=True)
    counts = np.bincount(np.asarray(be.sample(st, 400000, SplitMix64(7))), minlength=len(p))
    assert np.max(np.abs(counts / 400000 - p)) < 0.01


def test_cdf_and_alias_agree_statistically(be):
    # crates/qsv-core/src/sample.rs:234-258: device inverse-CDF vs the alias table
    w = np.array([0.25, 0.25, 0.4, 0.1])
    st = be.alloc(2)
    be.upload(st, np.sqrt(w), np.zeros(4))
    shots = 200000
    a = np.bincount(np.asarray(be.sample_alias(st, shots, SplitMix64(1))), minlength=4) / shots
    b = np.bincount(np.asarray(be.sample(st, shots, SplitMix64(2))), minlength=4) / shots
    assert np.max(np.abs(a - b)) < 0.01
    st.free()


def test_ghz_outcomes_and_determinism(be):
    n = 16
    st = be.alloc(n)
    be.init_basis(st, 0)
    be.run(st, ghz_chain(n))
    shots = 100000
    a = be.sample_device(st, shots, 7)
    assert set(np.unique(a).tolist()) == {0, (1 << n) - 1}
    ones = np.count_nonzero(a)
    assert abs(ones - shots / 2) < 5 * np.sqrt(shots / 4)
    assert np.array_equal(a, be.sample_device(st, shots, 7))
    assert not np.array_equal(a, be.sample_device(st, shots, 8))
    st.free()


def test_rejects_bad_shot_counts(be):
    st = be.alloc(4)
    be.init_basis(st, 3)
    out = np.zeros(1, dtype=np.uint64)
    assert L.lib().qsvb_sample(be.ctx, st.handle, 0, 1, out.ctypes.data_as(C.POINTER(C.c_uint64))) == L.QSVB_E_INVALID
    assert list(be.sample_device(st, 5, 1)) == [3] * 5
    st.free()
