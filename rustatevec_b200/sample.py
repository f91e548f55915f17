"""Host-side sampling primitives of the trait's default ``sample`` (crates/qsv-core/src/sample.rs).

``alias_sample`` builds Vose's alias table (sample.rs:33-82) and draws with two ``unit()`` values
per shot (sample.rs:84-97), consuming the SplitMix64 stream the same way the reference does.
"""
from __future__ import annotations

import numpy as np


def alias_table(weights):
    w = np.asarray(weights, dtype=np.float64)
    n = len(w)
    if n == 0:
        raise ValueError("AliasTable needs a non-empty distribution")
    total = float(w.sum())
    scaled = w * (n / total if total > 0 else 0.0)
    prob = np.zeros(n)
    alias = np.zeros(n, dtype=np.int64)
    small = [i for i in range(n) if scaled[i] < 1.0]
    large = [i for i in range(n) if scaled[i] >= 1.0]
    while small and large:
        s = small.pop()
        l = large.pop()
        prob[s] = scaled[s]
        alias[s] = l
        scaled[l] = (scaled[l] + scaled[s]) - 1.0
        (small if scaled[l] < 1.0 else large).append(l)
    for l in large:
        prob[l] = 1.0
    for s in small:
        prob[s] = 1.0
    return prob, alias


def alias_sample(weights, shots: int, rng) -> list:
    prob, alias = alias_table(weights)
    n = len(prob)
    out = []
    for _ in range(shots):
        i = min(int(rng.unit() * n), n - 1)
        out.append(i if rng.unit() < prob[i] else int(alias[i]))
    return out
