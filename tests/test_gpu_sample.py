"""Device sampling (qsvb_sample) against the same inverse-CDF rule computed on the host from the
state's FP64 probabilities with the reference's SplitMix64 stream (crates/qsv-core/src/circuits.rs:
22-46), plus the distribution checks of the reference's sampling tests
(crates/qsv-core/tests/sampling.rs: GHZ outcomes)."""
import ctypes as C

import numpy as np
import pytest

from rustatevec_b200 import B200Backend
from rustatevec_b200 import _lib as L
from rustatevec_b200.circuits import SplitMix64, ghz_chain, random_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["f64", "f32"])
def be(request, built):
    b = B200Backend(0, precision=request.param)
    yield b
    b.close()


def host_inverse_cdf(p, shots, seed):
    cdf = np.cumsum(p)
    rng = SplitMix64(seed)
    u = np.array([rng.unit() for _ in range(shots)]) * cdf[-1]
    idx = np.searchsorted(cdf, u, side="right")
    return np.minimum(idx, len(p) - 1)


@pytest.mark.parametrize("n", [6, 11, 18])
def test_matches_host_inverse_cdf(be, n):
    st = be.alloc(n)
    be.init_basis(st, 0)
    be.run(st, random_circuit(n, 10 * n, 40 + n))
    p = be.probabilities(st, fp64=True)
    shots = 20000
    got = be.sample_device(st, shots, 1234 + n)
    want = host_inverse_cdf(p, shots, 1234 + n)
    # the device sums in another order: only a draw within ~1e-15 of a boundary could differ
    assert np.count_nonzero(got != want) <= 1
    assert np.all(p[got.astype(np.int64)] > 0)
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
