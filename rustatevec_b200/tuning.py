"""Autotuning records and the learned cost model.

``collect`` runs the native autotuner (``qsvb_autotune``) on the device for a few state sizes and
precisions; ``train`` fits the MLP cost model on those records with the engine's own CUDA
forward/backward kernels (``qsvb_costmodel_train``) and installs it; ``save`` / ``load`` keep the
model image and the records as JSON. The planner uses the installed model for ``PLAN_LEARNED``
(fusion width, strategy, phase-run merging, CUDA-core vs tensor-core engine) and falls back to its
roofline model when none is installed.

Usage on a B200: ``python -m rustatevec_b200.tuning --out <model.json>``.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from . import _lib as L

NUM_FEATURES = 16
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200_costmodel.json")


def autotune(backend, n_qubits: int, reps: int = 3, seed: int = 0) -> dict:
    lib = L.lib()
    count = C.c_size_t(0)
    L.check(lib.qsvb_autotune(backend.ctx, n_qubits, backend.dtype, reps, seed, None, None, None, 0,
                              C.byref(count)))
    m = count.value
    feats = np.zeros((m, NUM_FEATURES), dtype=np.float32)
    secs = np.zeros(m, dtype=np.float64)
    kinds = np.zeros(m, dtype=np.uint32)
    L.check(lib.qsvb_autotune(backend.ctx, n_qubits, backend.dtype, reps, seed, feats.ctypes.data,
                              secs.ctypes.data, kinds.ctypes.data, m, C.byref(count)))
    return {"features": feats, "seconds": secs, "kinds": kinds,
            "n_qubits": np.full(m, n_qubits), "precision": [backend.precision] * m}


def plan_records(backend, n_qubits: int, reps: int = 2, seed: int = 0) -> dict:
    """Per-sweep device times of the candidate plans the planner weighs (qsv greedy fuse and window
    fusion at k = 2..6, CUDA-core and tensor-core engines) for representative circuits, so the model
    is trained on the sweeps real plans contain."""
    from .backend import Plan
    from .circuits import brickwork, qaoa_maxcut, qft, random_circuit
    circuits = [random_circuit(n_qubits, 20 * n_qubits, seed + 1), brickwork(n_qubits, 6, seed + 2),
                qft(n_qubits), qaoa_maxcut(n_qubits, 1, seed + 3)]
    engines = [L.ENGINE_CUDA_CORE] + ([L.ENGINE_TENSOR_CORE] if backend.dtype == L.C64 else [])
    feats, secs, kinds = [], [], []
    st = backend.alloc(n_qubits)
    try:
        backend.init_basis(st, 0)
        seen = set()
        for circ in circuits:
            for planner in (L.PLAN_GREEDY, L.PLAN_WINDOW):
                for k in (2, 4, 6):
                    for eng in engines:
                        p = Plan(backend, circ, L.make_opts(planner, k, eng, use_graph=False))
                        info = p.sweeps()
                        t = p.profile(st, reps)
                        for s, sec in zip(info, t):
                            key = tuple(s["features"])
                            if key in seen:
                                continue
                            seen.add(key)
                            feats.append(s["features"])
                            secs.append(sec)
                            kinds.append(L.SWEEP_KINDS.index(s["kind"]))
                        p.free()
    finally:
        st.free()
    m = len(secs)
    return {"features": np.asarray(feats, np.float32).reshape(m, NUM_FEATURES), "seconds": np.asarray(secs),
            "kinds": np.asarray(kinds, np.uint32), "n_qubits": np.full(m, n_qubits),
            "precision": [backend.precision] * m}


def collect(device: int = 0, sizes=(22, 25, 28, 30), precisions=("f32", "f64"), reps: int = 3) -> dict:
    from .backend import B200Backend
    parts = []
    for prec in precisions:
        be = B200Backend(device, precision=prec)
        try:
            for n in sizes:
                if prec == "f64" and n > 30:
                    continue
                parts.append(autotune(be, n, reps, seed=n))
                parts.append(plan_records(be, n, reps=2, seed=n))
        finally:
            be.close()
    return {k: (np.concatenate([p[k] for p in parts]) if k != "precision" else sum((p[k] for p in parts), []))
            for k in parts[0]}


def train(backend, records: dict, hidden: int = 64, epochs: int = 4000, lr: float = 3e-3, seed: int = 0) -> float:
    X = np.ascontiguousarray(records["features"], dtype=np.float32)
    y = np.ascontiguousarray(np.log2(records["seconds"]), dtype=np.float32)
    loss = C.c_float(0.0)
    L.check(L.lib().qsvb_costmodel_train(backend.ctx, X.ctypes.data, y.ctypes.data, len(y), hidden, epochs,
                                         lr, seed, C.byref(loss)))
    return float(loss.value)


def model_image() -> np.ndarray:
    need = C.c_size_t(0)
    L.check(L.lib().qsvb_costmodel_get(None, 0, C.byref(need)))
    img = np.zeros(need.value, dtype=np.float32)
    if need.value:
        L.check(L.lib().qsvb_costmodel_get(img.ctypes.data, need.value, C.byref(need)))
    return img


def install(image) -> None:
    if image is None or len(image) == 0:
        L.check(L.lib().qsvb_costmodel_set(None, 0))
        return
    img = np.ascontiguousarray(image, dtype=np.float32)
    L.check(L.lib().qsvb_costmodel_set(img.ctypes.data, len(img)))


def predict(features) -> np.ndarray:
    X = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, NUM_FEATURES)
    out = np.zeros(len(X), dtype=np.float32)
    L.check(L.lib().qsvb_costmodel_predict(X.ctypes.data, len(X), out.ctypes.data))
    return out


def save(path: str, records: dict | None = None, meta: dict | None = None) -> None:
    doc = {"model": model_image().tolist(), "meta": meta or {}}
    if records is not None:
        doc["records"] = {"features": records["features"].tolist(), "seconds": records["seconds"].tolist(),
                          "kinds": records["kinds"].tolist(), "n_qubits": records["n_qubits"].tolist(),
                          "precision": list(records["precision"])}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(doc, f)


def load(path: str = DEFAULT_MODEL) -> dict | None:
    """Install the model stored at ``path``; returns the document (None when absent)."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        doc = json.load(f)
    install(doc["model"])
    return doc


def records_from(doc: dict) -> dict:
    r = doc["records"]
    return {"features": np.asarray(r["features"], np.float32), "seconds": np.asarray(r["seconds"]),
            "kinds": np.asarray(r["kinds"], np.uint32), "n_qubits": np.asarray(r["n_qubits"]),
            "precision": list(r["precision"])}


def main():
    import argparse
    import time
    from .backend import B200Backend
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--sizes", default="22,25,28,30")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=4000)
    args = ap.parse_args()
    t0 = time.time()
    rec = collect(sizes=tuple(int(s) for s in args.sizes.split(",")), reps=args.reps)
    be = B200Backend(0, precision="f32")
    loss = train(be, rec, epochs=args.epochs)
    pred = predict(rec["features"])
    err = np.abs(pred - np.log2(rec["seconds"]))
    meta = {"records": int(len(rec["seconds"])), "final_loss": loss, "median_abs_log2_err": float(np.median(err)),
            "p90_abs_log2_err": float(np.quantile(err, 0.9)), "seconds": time.time() - t0}
    save(args.out, rec, meta)
    be.close()
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
