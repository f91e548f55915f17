"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates qsv's RefBackend, CpuBackend, fuse and reductions in C++
(oracle/qsv_oracle.cpp, which cites the reference lines it follows). Only the tests,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module, as the checker
and the timed CPU baseline; the product library never does.

Circuits are passed in the packed form ``(n_qubits, arity, qubits, mats)`` (any object with a
``flatten()`` method and ``n_qubits()`` works), matrices as interleaved FP64.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

REF, CPU_SERIAL, CPU_PARALLEL = 0, 1, 2
F32, F64 = 0, 1

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C")
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.orc_apply.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, f64p, u32p, C.c_uint32]
        L.orc_run.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_size_t, u32p, u32p, f64p]
        L.orc_fuse.argtypes = [C.c_int, C.c_uint32, C.c_size_t, u32p, u32p, f64p, u32p, u32p, f64p, C.c_size_t]
        L.orc_fuse.restype = C.c_long
        L.orc_gate.argtypes = [C.c_char_p, C.c_double, f64p, C.POINTER(C.c_uint32)]
        L.orc_is_diagonal.argtypes = [f64p, C.c_uint32]
        L.orc_expectation_z.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_uint64]
        L.orc_expectation_z.restype = C.c_double
        L.orc_norm_sqr.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint64]
        L.orc_norm_sqr.restype = C.c_double
        L.orc_probabilities.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
        for nm in ("orc_splitmix_next", "orc_splitmix_below"):
            getattr(L, nm).restype = C.c_uint64
        L.orc_splitmix_next.argtypes = [C.POINTER(C.c_uint64)]
        L.orc_splitmix_below.argtypes = [C.POINTER(C.c_uint64), C.c_uint64]
        L.orc_splitmix_unit.argtypes = [C.POINTER(C.c_uint64)]
        L.orc_splitmix_unit.restype = C.c_double
        for nm in ("orc_insert_zero_bit",):
            getattr(L, nm).restype = C.c_uint64
            getattr(L, nm).argtypes = [C.c_uint64, C.c_uint32]
        for nm in ("orc_insert_zero_bits", "orc_gather_bits", "orc_scatter_bits"):
            getattr(L, nm).restype = C.c_uint64
            getattr(L, nm).argtypes = [C.c_uint64, u32p, C.c_uint32]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def _np_dtype(dtype):
    return np.float64 if dtype == F64 else np.float32


def basis_state(n: int, dtype=F64, index: int = 0):
    """``StateVector::basis`` (crates/qsv-core/src/state/mod.rs:69-73) as SoA arrays."""
    re = np.zeros(1 << n, dtype=_np_dtype(dtype))
    im = np.zeros(1 << n, dtype=_np_dtype(dtype))
    re[index] = 1.0
    return re, im


def run(circuit, engine=REF, dtype=F64, state=None):
    """Run ``circuit`` from |0..0> (or from ``state`` = (re, im), copied) on the chosen oracle
    engine; returns ``(re, im)``."""
    n = circuit.n_qubits()
    if state is None:
        re, im = basis_state(n, dtype)
    else:
        re = np.array(state[0], dtype=_np_dtype(dtype), copy=True)
        im = np.array(state[1], dtype=_np_dtype(dtype), copy=True)
    arity, qubits, mats = circuit.flatten()
    rc = lib().orc_run(engine, dtype, n, re.ctypes.data, im.ctypes.data, len(arity), arity, qubits, mats)
    if rc:
        raise ValueError(f"oracle rejected the circuit (rc={rc})")
    return re, im


def apply(re, im, n, matrix, qubits, engine=REF):
    dtype = F64 if re.dtype == np.float64 else F32
    mat = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128)).reshape(-1).view(np.float64)
    qs = np.asarray(qubits, dtype=np.uint32)
    rc = lib().orc_apply(engine, dtype, n, re.ctypes.data, im.ctypes.data, np.ascontiguousarray(mat), qs, len(qs))
    if rc:
        raise ValueError("oracle rejected the gate")


def fuse(circuit, max_qubits, dtype=F64):
    """Reference ``fuse`` in precision R; returns ``(arity, qubits, mats)`` packed arrays."""
    arity, qubits, mats = circuit.flatten()
    n = len(arity)
    out_a = np.zeros(max(n, 1), np.uint32)
    out_q = np.zeros(max(int(arity.sum()) + 6 * n, 1), np.uint32)
    cap = max(2 * 4096 * max(n, 1), 16)
    out_m = np.zeros(cap, np.float64)
    k = lib().orc_fuse(dtype, max_qubits, n, arity, qubits, mats, out_a, out_q, out_m, cap)
    if k < 0:
        raise RuntimeError("oracle fuse buffer too small")
    a = out_a[:k].copy()
    nq = int(a.sum())
    nm = int(sum(2 * (1 << (2 * int(m))) for m in a))
    return a, out_q[:nq].copy(), out_m[:nm].copy()


def gate(name: str, theta: float = 0.0) -> np.ndarray:
    buf = np.zeros(32, np.float64)
    m = C.c_uint32(0)
    if lib().orc_gate(name.encode(), theta, buf, C.byref(m)):
        raise KeyError(name)
    d = 1 << m.value
    return buf[: 2 * d * d].view(np.complex128).reshape(d, d).copy()


def is_diagonal(matrix) -> bool:
    mat = np.ascontiguousarray(np.asarray(matrix, dtype=np.complex128))
    m = int(round(np.log2(mat.shape[0])))
    return bool(lib().orc_is_diagonal(np.ascontiguousarray(mat.reshape(-1).view(np.float64)), m))


def probabilities(re, im):
    dtype = F64 if re.dtype == np.float64 else F32
    out = np.empty_like(re)
    lib().orc_probabilities(dtype, re.ctypes.data, im.ctypes.data, len(re), out.ctypes.data)
    return out


def norm_sqr(re, im) -> float:
    dtype = F64 if re.dtype == np.float64 else F32
    return lib().orc_norm_sqr(dtype, re.ctypes.data, im.ctypes.data, len(re))


def expectation_z(probs, mask: int) -> float:
    dtype = F64 if probs.dtype == np.float64 else F32
    probs = np.ascontiguousarray(probs)
    return lib().orc_expectation_z(dtype, probs.ctypes.data, len(probs), mask)


def set_threads(n: int):
    lib().orc_set_threads(n)


_G = np.uint64(0x9E3779B97F4A7C15)


def splitmix_units(state: int, count: int) -> np.ndarray:
    """The next ``count`` ``unit()`` values of ``SplitMix64`` whose state is ``state``
    (crates/qsv-core/src/circuits.rs:22-46), vectorised: draw k mixes ``state + (k + 1) * G``."""
    k = np.arange(1, count + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(state) + k * _G
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def cdf_sample(weights, shots: int, state: int):
    """``cdf_sample`` (crates/qsv-core/src/sample.rs:163-172): the FP64 inclusive prefix sum of the
    weights, ``u = unit() * total`` per shot, and the first index whose cumulative value is
    ``>= u`` (``partition_point(|&c| c < u)``), clamped to the last index. The prefix sum is
    sequential (the reference's chunked parallel scan differs from it only by rounding). Returns
    ``(outcomes, u, cdf)``."""
    cdf = np.cumsum(np.asarray(weights, dtype=np.float64))
    u = splitmix_units(state, shots) * cdf[-1]
    idx = np.minimum(np.searchsorted(cdf, u, side="left"), len(cdf) - 1)
    return idx, u, cdf
