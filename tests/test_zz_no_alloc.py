"""The allocation-free <Z_mask> entry point (qsvb_expectation_z_noalloc).

Hosts that cannot let the library call cudaMalloc (a fixed device-memory budget, or a framework
that owns every device allocation through its own pool) call it on their own device buffers with
no context. This test gives it the device buffers of a state made the ordinary way and checks,
on two calls in a row, that it returns what qsvb_expectation_z returns and what numpy computes
from the downloaded amplitudes, within the parity tolerance of each precision. The file is named to run last, so a failure here does not hide
the rest of the suite; it also passes when run alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from rustatevec_b200 import B200Backend
from rustatevec_b200 import _lib as L
from rustatevec_b200.circuits import random_circuit

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "f32": 1e-5}


def device_buffers(state):
    n, dt = C.c_uint32(), C.c_int()
    re, im = C.c_void_p(), C.c_void_p()
    L.check(L.lib().qsvb_state_info(state.handle, C.byref(n), C.byref(dt), C.byref(re), C.byref(im)))
    return re, im, n.value, dt.value


def noalloc_expz(re, im, n, dtype, mask, stream):
    out = C.c_double(np.nan)
    rc = L.lib().qsvb_expectation_z_noalloc(re, im, n, dtype, mask, C.c_void_p(stream), C.byref(out))
    L.check(rc)
    return out.value


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_noalloc_matches_context_entry_point_twice(built, precision):
    be = B200Backend(0, precision=precision)
    try:
        c = random_circuit(14, 120, 2024)
        st = be.execute(c)
        re, im, n, dt = device_buffers(st)
        assert n == 14
        stream = be.stream()
        for mask in (1, 0b1011, (1 << 14) - 1, 0):
            want = be.expectation_z(st, mask)
            first = noalloc_expz(re, im, n, dt, mask, stream)
            second = noalloc_expz(re, im, n, dt, mask, stream)
            assert abs(first - want) <= TOL[precision], (mask, first, want)
            assert abs(second - want) <= TOL[precision], (mask, second, want)
        # mask 0 is the squared norm
        assert abs(noalloc_expz(re, im, n, dt, 0, 0) - be.norm_sqr(st)) <= TOL[precision]
        # and directly against numpy on the downloaded amplitudes
        psi = be.download(st).as_complex()
        for mask in (1, 0b1011, (1 << 14) - 1):
            assert abs(noalloc_expz(re, im, n, dt, mask, stream) - numpy_expz(psi, mask)) <= TOL[precision]
    finally:
        be.close()


def numpy_expz(psi, mask):
    """sum_i |psi_i|^2 (-1)^popcount(i & mask), in FP64 (crates/qsv-core/src/sample.rs:177-200)."""
    idx = np.arange(len(psi), dtype=np.uint64) & np.uint64(mask)
    parity = np.zeros(len(psi), dtype=np.uint64)
    while np.any(idx):
        parity ^= idx & np.uint64(1)
        idx >>= np.uint64(1)
    sign = 1.0 - 2.0 * parity.astype(np.float64)
    return float(np.sum(sign * np.abs(psi) ** 2))


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("n", [1, 2, 3])
def test_noalloc_small_states_against_numpy(built, precision, n):
    # the smallest states take the reduction's scalar branch
    be = B200Backend(0, precision=precision)
    try:
        rng = np.random.default_rng(n)
        v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
        v /= np.linalg.norm(v)
        st = be.alloc(n)
        be.upload(st, v.real, v.imag)
        psi = be.download(st).as_complex()
        re, im, _, dt = device_buffers(st)
        for mask in range(1 << n):
            want = numpy_expz(psi, mask)
            for _ in range(2):
                assert abs(noalloc_expz(re, im, n, dt, mask, 0) - want) <= TOL[precision], (n, mask)
    finally:
        be.close()


def test_noalloc_rejects_requests_beyond_its_limits(built):
    be = B200Backend(0, precision="f64")
    try:
        st = be.alloc(4)
        be.init_basis(st, 0)
        re, im, _, dt = device_buffers(st)
        out = C.c_double()
        lib = L.lib()
        assert lib.qsvb_expectation_z_noalloc(re, im, 35, dt, 1, None, C.byref(out)) == L.QSVB_E_INVALID
        assert "1..34" in lib.qsvb_last_error().decode()
        assert lib.qsvb_expectation_z_noalloc(re, im, 4, 7, 1, None, C.byref(out)) == L.QSVB_E_INVALID
        assert lib.qsvb_expectation_z_noalloc(None, im, 4, dt, 1, None, C.byref(out)) == L.QSVB_E_INVALID
        # a sub-buffer offset that breaks the 16-byte alignment, and host memory, are refused on
        # the host before any kernel is launched
        off8 = C.c_void_p(re.value + 8)
        assert lib.qsvb_expectation_z_noalloc(off8, im, 3, dt, 1, None, C.byref(out)) == L.QSVB_E_INVALID
        assert "aligned" in lib.qsvb_last_error().decode()
        host = np.zeros(64, dtype=np.float64)
        hp = C.c_void_p(host.ctypes.data + (-host.ctypes.data) % 16)
        assert lib.qsvb_expectation_z_noalloc(hp, im, 4, dt, 1, None, C.byref(out)) == L.QSVB_E_INVALID
        assert "device" in lib.qsvb_last_error().decode()
        # the library stays usable
        assert abs(noalloc_expz(re, im, 4, dt, 1, 0) - 1.0) < 1e-12
    finally:
        be.close()
