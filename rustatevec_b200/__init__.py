"""rustatevec_b200 — a B200-native statevector engine behind qsv's ``Backend`` trait.

The compute path is ``libqsvb.so`` (hand-written CUDA for sm_100a, C ABI in include/qsvb.h);
this package is its host-side mirror: gates, circuits, generators, fusion and the
``B200Backend`` that implements the trait's methods through the C ABI.
"""
from .gate import DenseGate
from .circuit import Circuit, GateOp
from .circuits import SplitMix64, ghz, qft, random_circuit
from .fusion import FusionConfig, fuse
from ._lib import (C64, C128, PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_WINDOW, PLAN_LEARNED, PLAN_TILE, PLAN_CHAIN,
                   ENGINE_AUTO, ENGINE_CUDA_CORE, ENGINE_TENSOR_CORE, QsvbError)
from .backend import B200Backend, DeviceState, Plan, StateVector

__all__ = [
    "DenseGate", "Circuit", "GateOp", "SplitMix64", "ghz", "qft", "random_circuit",
    "FusionConfig", "fuse", "B200Backend", "DeviceState", "Plan", "StateVector", "QsvbError",
    "C64", "C128", "PLAN_AS_GIVEN", "PLAN_GREEDY", "PLAN_WINDOW", "PLAN_LEARNED", "PLAN_TILE", "PLAN_CHAIN",
    "ENGINE_AUTO", "ENGINE_CUDA_CORE", "ENGINE_TENSOR_CORE",
]
