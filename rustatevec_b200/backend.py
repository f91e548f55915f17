"""``B200Backend`` — qsv's ``Backend<R>`` trait served by the CUDA engine.

Method for method this mirrors ``trait Backend<R>`` (crates/qsv-core/src/backend/mod.rs:31-74):

========================  ============================================================
trait method              here
========================  ============================================================
``alloc(n)``              ``qsvb_state_alloc`` (device SoA re/im; contents unspecified)
``init_basis(s, b)``      ``qsvb_init_basis``
``apply(s, gate, qs)``    ``qsvb_apply`` (diagonal / butterfly / controlled / dense fast paths)
``amplitude(s, i)``       ``qsvb_amplitude`` (one element, not the whole state)
``probabilities(s)``      ``qsvb_probabilities`` (FP64 on device, returned in R)
``sample(s, shots, rng)`` ``qsvb_sample``: inverse-CDF draws on the device (cdf_sample, sample.rs:163-172)
``expectation_z(s, m)``   ``qsvb_expectation_z`` (FP64 on device)
``download(s)``           ``qsvb_download`` -> host ``StateVector``
``execute(circuit)``      alloc + init_basis(0) + ``qsvb_execute`` (planned, sweeps launched directly)
========================  ============================================================

``R`` is chosen per backend instance: ``B200Backend(precision="f64")`` serves complex128 states
(``Backend<f64>``), ``precision="f32"`` complex64 (``Backend<f32>``). Errors raise ``QsvbError``
where the Rust trait would panic.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .circuit import Circuit
from .gate import DenseGate


class StateVector:
    """Host SoA statevector, the ``download`` target (crates/qsv-core/src/state/mod.rs:25-134)."""

    def __init__(self, re: np.ndarray, im: np.ndarray):
        self.re = re
        self.im = im

    def n_qubits(self) -> int:
        return int(self.re.shape[0]).bit_length() - 1

    def dim(self) -> int:
        return int(self.re.shape[0])

    def amplitude(self, i: int) -> complex:
        return complex(self.re[i], self.im[i])

    def as_complex(self) -> np.ndarray:
        return self.re.astype(np.float64) + 1j * self.im.astype(np.float64)

    def norm_sqr(self) -> float:
        return float(np.sum(self.re.astype(np.float64) ** 2 + self.im.astype(np.float64) ** 2))

    def probabilities(self) -> np.ndarray:
        return self.re * self.re + self.im * self.im


class DeviceState:
    """Opaque device-resident state (the trait's ``type State``); freed with the object."""

    def __init__(self, backend: "B200Backend", handle: C.c_void_p, n_qubits: int):
        self._backend = backend
        self.handle = handle
        self.n = n_qubits

    def n_qubits(self) -> int:
        return self.n

    def free(self):
        if self.handle:
            L.check(L.lib().qsvb_state_free(self._backend.ctx, self.handle))
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self._backend.ctx:
                L.lib().qsvb_state_free(self._backend.ctx, self.handle)
                self.handle = None
        except Exception:
            pass


class B200Backend:
    def __init__(self, device: int = 0, precision: str = "f64", planner: int = L.PLAN_GREEDY,
                 max_fused_qubits: int = 4, engine: int = L.ENGINE_AUTO, use_graph: bool = True):
        if precision not in ("f32", "f64"):
            raise ValueError("precision must be 'f32' or 'f64'")
        self.precision = precision
        self.dtype = L.C128 if precision == "f64" else L.C64
        self.np_real = np.float64 if precision == "f64" else np.float32
        self.opts = L.make_opts(planner, max_fused_qubits, engine, use_graph)
        self.last_stats = None
        h = C.c_void_p()
        self.ctx = None
        L.check(L.lib().qsvb_create(device, C.byref(h)))
        self.ctx = h

    def close(self):
        if self.ctx:
            L.check(L.lib().qsvb_destroy(self.ctx))
            self.ctx = None

    def __del__(self):
        try:
            if self.ctx:
                L.lib().qsvb_destroy(self.ctx)
                self.ctx = None
        except Exception:
            pass

    # ---- trait methods
    def alloc(self, n_qubits: int) -> DeviceState:
        h = C.c_void_p()
        L.check(L.lib().qsvb_state_alloc(self.ctx, n_qubits, self.dtype, C.byref(h)))
        return DeviceState(self, h, n_qubits)

    def init_basis(self, state: DeviceState, basis: int):
        L.check(L.lib().qsvb_init_basis(self.ctx, state.handle, basis))

    def apply(self, state: DeviceState, gate: DenseGate, qubits):
        qs = np.ascontiguousarray(np.asarray(qubits, dtype=np.uint32))
        mat = np.ascontiguousarray(gate.matrix.reshape(-1).view(np.float64))
        L.check(L.lib().qsvb_apply(self.ctx, state.handle, mat.ctypes.data_as(L._dp),
                                   qs.ctypes.data_as(C.POINTER(C.c_uint32)), len(qs)))

    def amplitude(self, state: DeviceState, index: int) -> complex:
        out = (C.c_double * 2)()
        L.check(L.lib().qsvb_amplitude(self.ctx, state.handle, index, out))
        return complex(out[0], out[1])

    def probabilities(self, state: DeviceState, fp64: bool = False) -> np.ndarray:
        dt = np.float64 if (fp64 or self.dtype == L.C128) else np.float32
        out = np.empty(1 << state.n, dtype=dt)
        L.check(L.lib().qsvb_probabilities(self.ctx, state.handle, out.ctypes.data,
                                           L.C128 if dt == np.float64 else L.C64))
        return out

    def sample(self, state: DeviceState, shots: int, rng) -> list:
        """``Backend::sample`` (mod.rs:52-54) overridden on the device, as the trait's doc asks of a
        device backend: inverse-CDF draws (cdf_sample, sample.rs:163-172) from ``rng``'s stream,
        one ``unit()`` per shot, with no probability download; ``rng`` advances by ``shots`` draws.
        """
        out = self.sample_device(state, shots, rng.state)
        rng.state = (rng.state + shots * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        return [int(x) for x in out]

    def sample_alias(self, state: DeviceState, shots: int, rng) -> list:
        """The trait's default body (mod.rs:52-54): Vose alias sampling (sample.rs:84-97) over the
        downloaded FP64 probabilities, two ``unit()`` per shot. Same distribution as ``sample``,
        other draws; it downloads 2^n probabilities, so it suits small states only."""
        from .sample import alias_sample
        return alias_sample(self.probabilities(state, fp64=True), shots, rng)

    def sample_device(self, state: DeviceState, shots: int, seed: int) -> np.ndarray:
        """``shots`` outcomes drawn on the device by inverse-CDF sampling (qsvb_sample): shot k uses
        the k-th ``unit()`` of ``SplitMix64(seed)`` and takes the first outcome whose cumulative
        probability reaches ``unit() * total``; no probability download."""
        out = np.empty(shots, dtype=np.uint64)
        L.check(L.lib().qsvb_sample(self.ctx, state.handle, shots, seed,
                                    out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    def expectation_z(self, state: DeviceState, mask: int) -> float:
        out = C.c_double()
        L.check(L.lib().qsvb_expectation_z(self.ctx, state.handle, mask, C.byref(out)))
        return out.value

    def norm_sqr(self, state: DeviceState) -> float:
        out = C.c_double()
        L.check(L.lib().qsvb_norm_sqr(self.ctx, state.handle, C.byref(out)))
        return out.value

    def inner_product(self, a: DeviceState, b: DeviceState) -> complex:
        out = (C.c_double * 2)()
        L.check(L.lib().qsvb_inner_product(self.ctx, a.handle, b.handle, out))
        return complex(out[0], out[1])

    def fidelity(self, a: DeviceState, b: DeviceState) -> float:
        out = C.c_double()
        L.check(L.lib().qsvb_fidelity(self.ctx, a.handle, b.handle, C.byref(out)))
        return out.value

    def download(self, state: DeviceState) -> StateVector:
        re = np.empty(1 << state.n, dtype=self.np_real)
        im = np.empty(1 << state.n, dtype=self.np_real)
        L.check(L.lib().qsvb_download(self.ctx, state.handle, re.ctypes.data, im.ctypes.data))
        return StateVector(re, im)

    def upload(self, state: DeviceState, re, im):
        re = np.ascontiguousarray(re, dtype=self.np_real)
        im = np.ascontiguousarray(im, dtype=self.np_real)
        L.check(L.lib().qsvb_upload(self.ctx, state.handle, re.ctypes.data, im.ctypes.data))

    def init_gaussian(self, state: DeviceState, seed: int):
        L.check(L.lib().qsvb_init_gaussian(self.ctx, state.handle, seed))

    def run(self, state: DeviceState, circuit: Circuit, opts=None) -> dict:
        """Queue ``circuit`` on an initialised ``state`` (the body of ``execute``)."""
        pc = L.PackedCircuit(circuit)
        st = L.PlanStats()
        L.check(L.lib().qsvb_execute(self.ctx, state.handle, pc.ref(), C.byref(opts or self.opts),
                                     C.byref(st)))
        self.last_stats = st.to_dict()
        return self.last_stats

    def execute(self, circuit: Circuit) -> DeviceState:
        """``Backend::execute`` (mod.rs:66-73): alloc, |0..0>, then the whole circuit."""
        state = self.alloc(circuit.n_qubits())
        self.init_basis(state, 0)
        self.run(state, circuit)
        return state

    def execute_batch(self, circuits, probabilities: bool = True, local_qubits: int = 0, register_qubits: int = 0):
        """Run many small circuits (each from |0..0>) in one persistent kernel: the batched form of
        ``execute`` followed by ``expectation_z(probs, 1)`` (sample.rs:177-200) per circuit.

        Returns ``(z0, probs, stats)``: ``z0`` f64[count]; ``probs`` one FP64 array of 2^n_i per
        circuit (views into one packed buffer) or None; ``stats`` the batch statistics with
        ``measured_seconds`` = measured device seconds."""
        pb = circuits if isinstance(circuits, L.PackedBatch) else L.PackedBatch(circuits)
        z0 = np.zeros(pb.count, dtype=np.float64)
        probs = None
        pptr = None
        if probabilities:
            sizes = np.left_shift(1, pb.n_qubits)
            probs_flat = np.empty(int(sizes.sum()), dtype=np.float64)
            pptr = probs_flat.ctypes.data_as(C.POINTER(C.c_double))
        st = L.PlanStats()
        L.check(L.lib().qsvb_execute_batch_ex(self.ctx, pb.ptr(), pb.count, self.dtype, local_qubits,
                                              register_qubits, z0.ctypes.data_as(C.POINTER(C.c_double)), pptr, None,
                                              C.byref(st)))
        if probabilities:
            edges = np.concatenate([[0], np.cumsum(sizes)])
            probs = [probs_flat[edges[i]:edges[i + 1]] for i in range(pb.count)]
        return z0, probs, st.to_dict()

    def stream(self) -> int:
        """The engine's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        out = C.c_void_p()
        L.check(L.lib().qsvb_stream(self.ctx, C.byref(out)))
        return int(out.value or 0)

    def synchronize(self):
        L.check(L.lib().qsvb_synchronize(self.ctx))


class Plan:
    """A reusable execution plan (``qsvb_plan_*``): plan once, run many times."""

    def __init__(self, backend: B200Backend, circuit: Circuit, opts=None):
        self.backend = backend
        self._pc = L.PackedCircuit(circuit)
        h = C.c_void_p()
        L.check(L.lib().qsvb_plan_create(backend.ctx, self._pc.ref(), backend.dtype,
                                         C.byref(opts or backend.opts), C.byref(h)))
        self.handle = h

    def run(self, state: DeviceState):
        L.check(L.lib().qsvb_plan_run(self.backend.ctx, self.handle, state.handle))

    def stats(self) -> dict:
        st = L.PlanStats()
        L.check(L.lib().qsvb_plan_stats_get(self.handle, C.byref(st)))
        return st.to_dict()

    def sweeps(self) -> list:
        out = []
        for i in range(self.stats()["n_sweeps"]):
            si = L.SweepInfo()
            L.check(L.lib().qsvb_plan_sweep_info(self.handle, i, C.byref(si)))
            out.append(si.to_dict())
        return out

    def profile(self, state: DeviceState, reps: int = 3) -> np.ndarray:
        """Mean device seconds per launch of each sweep (CUDA events, native)."""
        n = self.stats()["n_sweeps"]
        out = np.zeros(max(n, 1), dtype=np.float64)
        L.check(L.lib().qsvb_plan_profile(self.backend.ctx, self.handle, state.handle, reps,
                                          out.ctypes.data_as(L._dp)))
        return out[:n]

    def free(self):
        if self.handle:
            L.check(L.lib().qsvb_plan_free(self.backend.ctx, self.handle))
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.backend.ctx:
                L.lib().qsvb_plan_free(self.backend.ctx, self.handle)
                self.handle = None
        except Exception:
            pass
