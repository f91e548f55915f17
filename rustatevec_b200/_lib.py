"""ctypes binding of libqsvb.so (the C ABI declared in include/qsvb.h).

The shared library is built in-tree (``rustatevec_b200/libqsvb.so``) by
``__graft_entry__.build()`` / ``make -C rustatevec_b200/csrc``. There is no fallback: if the
library is missing or fails to load, importing the backend raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# QSVB_LIBRARY selects another build of the engine, e.g. the bounds-checked libqsvb_checked.so
# (`make -C rustatevec_b200/csrc BOUNDS=1`)
LIB_PATH = os.environ.get("QSVB_LIBRARY") or os.path.join(_HERE, "libqsvb.so")

QSVB_OK = 0
QSVB_E_INVALID = -1
QSVB_E_CUDA = -2
QSVB_E_OOM = -3
QSVB_E_UNSUPPORTED = -4
QSVB_E_TIMEOUT = -5

C64, C128 = 0, 1
PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_WINDOW, PLAN_LEARNED, PLAN_TILE, PLAN_CHAIN = 0, 1, 2, 3, 4, 5
ENGINE_AUTO, ENGINE_CUDA_CORE, ENGINE_TENSOR_CORE = 0, 1, 2
MAX_GATE_QUBITS = 6

SWEEP_KINDS = ("1q", "ctrl1q", "diag", "phase", "dense", "dense_tc", "tile", "other", "tc_chain", "permute")


class QsvbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"qsvb error {code}: {msg}")
        self.code = code


class Gate(C.Structure):
    _fields_ = [("n_qubits", C.c_uint32), ("qubits", C.c_uint32 * MAX_GATE_QUBITS),
                ("matrix", C.POINTER(C.c_double))]


class CircuitS(C.Structure):
    _fields_ = [("n_qubits", C.c_uint32), ("n_gates", C.c_size_t), ("gates", C.POINTER(Gate))]


class PlanOpts(C.Structure):
    _fields_ = [("planner", C.c_uint32), ("max_fused_qubits", C.c_uint32), ("engine", C.c_uint32),
                ("use_graph", C.c_uint32), ("chain_max_matrices", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class PlanStats(C.Structure):
    _fields_ = [("n_gates_in", C.c_uint64), ("n_sweeps", C.c_uint64),
                ("n_sweeps_by_kind", C.c_uint64 * 10), ("algorithmic_bytes", C.c_double),
                ("full_sweep_bytes", C.c_double), ("flops", C.c_double),
                ("predicted_seconds", C.c_double), ("measured_seconds", C.c_double)]

    def to_dict(self) -> dict:
        return {
            "n_gates_in": int(self.n_gates_in), "n_sweeps": int(self.n_sweeps),
            "by_kind": {k: int(v) for k, v in zip(SWEEP_KINDS, self.n_sweeps_by_kind) if v},
            "algorithmic_bytes": float(self.algorithmic_bytes),
            "full_sweep_bytes": float(self.full_sweep_bytes), "flops": float(self.flops),
            "predicted_seconds": float(self.predicted_seconds),
            "measured_seconds": float(self.measured_seconds),
        }


class SweepInfo(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("n_qubits", C.c_uint32), ("qubits", C.c_uint32 * MAX_GATE_QUBITS),
                ("target", C.c_uint32), ("n_ctrl", C.c_uint32), ("ctrl", C.c_uint32 * MAX_GATE_QUBITS),
                ("n_terms", C.c_uint32), ("n_gates", C.c_uint64), ("algorithmic_bytes", C.c_double),
                ("flops", C.c_double), ("features", C.c_float * 16)]

    def to_dict(self) -> dict:
        return {"kind": SWEEP_KINDS[self.kind], "k": int(self.n_qubits),
                "qubits": [int(self.qubits[j]) for j in range(self.n_qubits)],
                "target": int(self.target), "ctrl": [int(self.ctrl[j]) for j in range(self.n_ctrl)],
                "n_terms": int(self.n_terms), "n_gates": int(self.n_gates),
                "algorithmic_bytes": float(self.algorithmic_bytes), "flops": float(self.flops),
                "features": [float(x) for x in self.features]}


# Every exported symbol, with (restype, argtypes). Kept in the order of include/qsvb.h.
_vp, _u32, _u64, _i, _sz, _d = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_size_t, C.c_double
_dp = C.POINTER(C.c_double)
SIGNATURES = {
    "qsvb_create": (_i, [_i, C.POINTER(_vp)]),
    "qsvb_destroy": (_i, [_vp]),
    "qsvb_last_error": (C.c_char_p, []),
    "qsvb_synchronize": (_i, [_vp]),
    "qsvb_version": (C.c_char_p, []),
    "qsvb_stream": (_i, [_vp, C.POINTER(_vp)]),
    "qsvb_state_alloc": (_i, [_vp, _u32, _i, C.POINTER(_vp)]),
    "qsvb_state_free": (_i, [_vp, _vp]),
    "qsvb_state_info": (_i, [_vp, C.POINTER(_u32), C.POINTER(_i), C.POINTER(_vp), C.POINTER(_vp)]),
    "qsvb_init_basis": (_i, [_vp, _vp, _u64]),
    "qsvb_upload": (_i, [_vp, _vp, _vp, _vp]),
    "qsvb_init_gaussian": (_i, [_vp, _vp, _u64]),
    "qsvb_apply": (_i, [_vp, _vp, _dp, C.POINTER(_u32), _u32]),
    "qsvb_execute": (_i, [_vp, _vp, C.POINTER(CircuitS), C.POINTER(PlanOpts), C.POINTER(PlanStats)]),
    "qsvb_plan_create": (_i, [_vp, C.POINTER(CircuitS), _i, C.POINTER(PlanOpts), C.POINTER(_vp)]),
    "qsvb_plan_run": (_i, [_vp, _vp, _vp]),
    "qsvb_plan_stats_get": (_i, [_vp, C.POINTER(PlanStats)]),
    "qsvb_plan_free": (_i, [_vp, _vp]),
    "qsvb_plan_sweep_info": (_i, [_vp, _sz, C.c_void_p]),
    "qsvb_plan_profile": (_i, [_vp, _vp, _vp, _i, _dp]),
    "qsvb_plan_dry_run": (_i, [C.POINTER(CircuitS), _i, C.POINTER(PlanOpts), C.POINTER(PlanStats)]),
    "qsvb_fuse": (_i, [C.POINTER(CircuitS), C.POINTER(PlanOpts), C.POINTER(Gate), C.POINTER(_sz), _dp, _sz]),
    "qsvb_download": (_i, [_vp, _vp, _vp, _vp]),
    "qsvb_amplitude": (_i, [_vp, _vp, _u64, _dp]),
    "qsvb_probabilities": (_i, [_vp, _vp, _vp, _i]),
    "qsvb_expectation_z": (_i, [_vp, _vp, _u64, _dp]),
    "qsvb_sample": (_i, [_vp, _vp, _u64, _u64, C.POINTER(_u64)]),
    "qsvb_norm_sqr": (_i, [_vp, _vp, _dp]),
    "qsvb_inner_product": (_i, [_vp, _vp, _vp, _dp]),
    "qsvb_fidelity": (_i, [_vp, _vp, _vp, _dp]),
    "qsvb_expectation_z_noalloc": (_i, [_vp, _vp, _u32, _i, _u64, _vp, _dp]),
    "qsvb_autotune": (_i, [_vp, _u32, _i, _i, _u64, C.c_void_p, C.c_void_p, C.c_void_p, _sz, C.POINTER(_sz)]),
    "qsvb_costmodel_train": (_i, [_vp, C.c_void_p, C.c_void_p, _sz, _u32, _u32, C.c_float, _u64,
                                  C.POINTER(C.c_float)]),
    "qsvb_costmodel_forward_backward": (_i, [_vp, C.c_void_p, _u32, C.c_void_p, C.c_void_p, _sz,
                                             C.POINTER(C.c_float), C.c_void_p]),
    "qsvb_costmodel_get": (_i, [C.c_void_p, _sz, C.POINTER(_sz)]),
    "qsvb_costmodel_set": (_i, [C.c_void_p, _sz]),
    "qsvb_costmodel_predict": (_i, [C.c_void_p, _sz, C.c_void_p]),
    "qsvb_execute_batch": (_i, [_vp, C.POINTER(CircuitS), _sz, _i, _dp, _dp, C.POINTER(_u64),
                                C.POINTER(PlanStats)]),
    "qsvb_batch_create": (_i, [_vp, C.POINTER(CircuitS), _sz, _i, _u32, _u32, C.POINTER(_vp)]),
    "qsvb_batch_run": (_i, [_vp, _vp, _dp, _dp, C.POINTER(_u64), C.POINTER(PlanStats)]),
    "qsvb_batch_free": (_i, [_vp, _vp]),
    "qsvb_batch_set_wait_budget": (_i, [_vp, _vp, _u64]),
    "qsvb_batch_autotune": (_i, [_vp, C.POINTER(CircuitS), _sz, _i, C.POINTER(_u32), C.POINTER(_u32), _dp, _sz,
                                 C.POINTER(_sz)]),
    "qsvb_execute_batch_ex": (_i, [_vp, C.POINTER(CircuitS), _sz, _i, _u32, _u32, _dp, _dp, C.POINTER(_u64),
                                   C.POINTER(PlanStats)]),
}

_lib = None


def lib():
    """Load libqsvb.so (once). Raises if it is missing: there is no CPU fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C rustatevec_b200/csrc` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != QSVB_OK:
        raise QsvbError(rc, lib().qsvb_last_error().decode(errors="replace"))


class PackedCircuit:
    """A circuit packed into the C structs; keeps the matrix buffer alive."""

    def __init__(self, circuit):
        arity, qubits, mats = circuit.flatten()
        self.mats = np.ascontiguousarray(mats, dtype=np.float64)
        n = len(arity)
        self.gates = (Gate * max(n, 1))()
        base = self.mats.ctypes.data
        qo = mo = 0
        for i, m in enumerate(arity.tolist()):
            g = self.gates[i]
            g.n_qubits = m
            for j in range(m):
                g.qubits[j] = int(qubits[qo + j])
            g.matrix = C.cast(base + 8 * mo, _dp)
            qo += m
            mo += 2 * (1 << (2 * m))
        self.struct = CircuitS(circuit.n_qubits(), n, C.cast(self.gates, C.POINTER(Gate)))

    def ref(self):
        """By-reference argument for the C calls. The struct points into this object's gate array
        and matrix buffer: keep the PackedCircuit alive until the call returns."""
        return C.byref(self.struct)


_GATE_DT = np.dtype({"names": ["n", "q", "mat"], "formats": ["<u4", ("<u4", MAX_GATE_QUBITS), "<u8"],
                     "offsets": [0, 4, 32], "itemsize": 40})
_CIRC_DT = np.dtype({"names": ["n", "ngates", "gates"], "formats": ["<u4", "<u8", "<u8"],
                     "offsets": [0, 8, 16], "itemsize": 24})


class PackedBatch:
    """Many circuits packed into one ``qsvb_circuit`` array (numpy-built, no per-gate Python
    ctypes work); keeps every buffer alive."""

    def __init__(self, circuits):
        assert C.sizeof(Gate) == _GATE_DT.itemsize and C.sizeof(CircuitS) == _CIRC_DT.itemsize
        from itertools import chain
        from .circuit import flatten_ops
        counts = np.array([len(c) for c in circuits], dtype=np.int64)
        arity, allq, mats = flatten_ops(list(chain.from_iterable(c.ops() for c in circuits)))
        self.mats = mats if len(mats) else np.zeros(1)
        ng = len(arity)
        self.gates = np.zeros(max(ng, 1), dtype=_GATE_DT)
        self.gates["n"][:ng] = arity
        a64 = arity.astype(np.int64)
        qoff = np.concatenate([[0], np.cumsum(a64)])
        for j in range(int(a64.max()) if ng else 0):
            sel = a64 > j
            self.gates["q"][:ng][sel, j] = allq[qoff[:-1][sel] + j]
        moff = np.concatenate([[0], np.cumsum(2 * (1 << (2 * a64)))])[:-1]
        self.gates["mat"][:ng] = self.mats.ctypes.data + 8 * moff
        nc = len(circuits)
        goff = np.concatenate([[0], np.cumsum(counts)])[:-1]
        self.circs = np.zeros(max(nc, 1), dtype=_CIRC_DT)
        self.circs["n"][:nc] = [c.n_qubits() for c in circuits]
        self.circs["ngates"][:nc] = counts
        self.circs["gates"][:nc] = self.gates.ctypes.data + _GATE_DT.itemsize * goff
        self.count = nc
        self.n_qubits = np.array([c.n_qubits() for c in circuits], dtype=np.int64)

    def ptr(self):
        """Pointer argument for the C calls; keep the PackedBatch alive until the call returns."""
        return C.cast(self.circs.ctypes.data, C.POINTER(CircuitS))


def make_opts(planner=PLAN_GREEDY, max_fused_qubits=4, engine=ENGINE_AUTO, use_graph=True,
              chain_max_matrices=0) -> PlanOpts:
    o = PlanOpts()
    o.planner = planner
    o.max_fused_qubits = max_fused_qubits
    o.engine = engine
    o.use_graph = 1 if use_graph else 0
    o.chain_max_matrices = chain_max_matrices
    return o
