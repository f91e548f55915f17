"""The allocation-free <Z_mask> entry point (qsvb_expectation_z_noalloc).

Hosts that cannot let the library call cudaMalloc (a fixed device-memory budget, or a framework
that owns every device allocation through its own pool) call it on their own device buffers with
no context. This test gives it the device buffers of a state made the ordinary way and checks,
on two calls in a row, that it returns what qsvb_expectation_z returns, within the parity
tolerance of each precision. The file is named to run last, so a failure here does not hide
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
        # the library stays usable
        assert abs(noalloc_expz(re, im, 4, dt, 1, 0) - 1.0) < 1e-12
    finally:
        be.close()
