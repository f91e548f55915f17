"""Circuit generators and the deterministic RNG.

``SplitMix64``, ``ghz``, ``qft`` and ``random_circuit`` mirror qsv's ``circuits.rs``
(crates/qsv-core/src/circuits.rs:12-113) and consume the random stream in the same order, so
the same seed gives the same circuit as the reference.

The workload generators below (``ghz_chain``, ``brickwork``, ``qaoa_maxcut``,
``ansatz_batch``) have no counterpart in the reference; they define the benchmark
configurations on top of the same RNG. Choices the reference leaves open are fixed here:

* Haar SU(2): four standard normals from two Box-Muller pairs (each uniform drawn with
  ``unit()``), normalised to a unit quaternion ``(a, b, c, d)`` and mapped to
  ``[[a+ib, c+id], [-c+id, a-ib]]``.
* The ansatz layer ``RY(theta) RZ(phi)`` is read as an operator product: RZ is applied first.
* QAOA graph: a 3-regular graph on an odd node count does not exist, so for odd ``n`` node 0
  gets degree 4 and every other node degree 3 (configuration model on SplitMix64 with
  rejection of self loops and multi-edges). The start state is ``|+>^n`` (H on every qubit);
  each cost layer is ``RZZ(-gamma)`` on every edge (``exp(-i gamma C)`` for the MaxCut cost up to a
  global phase) and each mixer is ``RX(2 beta)`` on every qubit.
"""
from __future__ import annotations

import math

from .circuit import Circuit
from . import gate as G

_MASK = (1 << 64) - 1


class SplitMix64:
    """SplitMix64 (circuits.rs:12-48)."""

    def __init__(self, seed: int):
        self.state = seed & _MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        return self.next_u64() % n

    def unit(self) -> float:
        return (self.next_u64() >> 11) / float(1 << 53)

    def angle(self) -> float:
        return self.unit() * (2.0 * math.pi)

    def normal(self) -> tuple:
        """Two independent standard normals (Box-Muller)."""
        u1 = 1.0 - self.unit()  # (0, 1]
        u2 = self.unit()
        r = math.sqrt(-2.0 * math.log(u1))
        return r * math.cos(2.0 * math.pi * u2), r * math.sin(2.0 * math.pi * u2)


def ghz(n: int) -> Circuit:
    """``H(0); CX(0, q)`` for q = 1..n (circuits.rs:50-57)."""
    c = Circuit(n)
    c.h(0)
    for q in range(1, n):
        c.cx(0, q)
    return c


def qft(n: int) -> Circuit:
    """Hadamards + controlled phases + final swaps (circuits.rs:61-74)."""
    c = Circuit(n)
    for j in range(n):
        c.h(j)
        for k in range(j + 1, n):
            c.cphase(k, j, math.pi / float(1 << (k - j)))
    for j in range(n // 2):
        c.swap(j, n - 1 - j)
    return c


def random_circuit(n_qubits: int, n_gates: int, seed: int) -> Circuit:
    """Seeded random circuit over the full 1q/2q gate set (circuits.rs:79-113)."""
    if n_qubits < 2:
        raise ValueError("random_circuit needs at least 2 qubits")
    rng = SplitMix64(seed)
    c = Circuit(n_qubits)
    one_q = [c.h, c.x, c.y, c.z, c.s, c.t, c.sx]
    for _ in range(n_gates):
        q = rng.below(n_qubits)
        k = rng.below(15)
        if k < 7:
            one_q[k](q)
        elif k == 7:
            c.rx(q, rng.angle())
        elif k == 8:
            c.ry(q, rng.angle())
        elif k == 9:
            c.rz(q, rng.angle())
        elif k == 10:
            c.phase(q, rng.angle())
        else:
            q2 = rng.below(n_qubits)
            while q2 == q:
                q2 = rng.below(n_qubits)
            k2 = rng.below(4)
            if k2 == 0:
                c.cx(q, q2)
            elif k2 == 1:
                c.cz(q, q2)
            elif k2 == 2:
                c.swap(q, q2)
            else:
                c.rzz(q, q2, rng.angle())
    return c


# ----------------------------------------------------------------- benchmark workloads

def ghz_chain(n: int) -> Circuit:
    """GHZ by a CX chain: ``H(0)`` then ``CX(i, i+1)`` for i = 0..n-2 (n gates)."""
    c = Circuit(n)
    c.h(0)
    for i in range(n - 1):
        c.cx(i, i + 1)
    return c


def haar_su2(rng: SplitMix64):
    z0, z1 = rng.normal()
    z2, z3 = rng.normal()
    nrm = math.sqrt(z0 * z0 + z1 * z1 + z2 * z2 + z3 * z3)
    return G.u_from_quaternion(z0 / nrm, z1 / nrm, z2 / nrm, z3 / nrm)


def brickwork(n: int, depth: int, seed: int) -> Circuit:
    """Random brickwork: per layer a Haar SU(2) on every qubit, then CZ(i, i+1) for i even on
    even layers and i odd on odd layers."""
    rng = SplitMix64(seed)
    c = Circuit(n)
    for layer in range(depth):
        for q in range(n):
            c.push(haar_su2(rng), [q])
        for i in range(layer % 2, n - 1, 2):
            c.cz(i, i + 1)
    return c


def regular_graph(n: int, seed: int, degree: int = 3):
    """Seeded random graph: every node of degree ``degree``; when ``n * degree`` is odd, node 0
    gets one extra stub. Configuration model with rejection (no loops, no multi-edges)."""
    rng = SplitMix64(seed)
    deg = [degree] * n
    if (n * degree) % 2:
        deg[0] += 1
    for _attempt in range(10000):
        stubs = [v for v in range(n) for _ in range(deg[v])]
        for i in range(len(stubs) - 1, 0, -1):
            j = rng.below(i + 1)
            stubs[i], stubs[j] = stubs[j], stubs[i]
        edges = set()
        ok = True
        for i in range(0, len(stubs), 2):
            a, b = stubs[i], stubs[i + 1]
            if a == b or (min(a, b), max(a, b)) in edges:
                ok = False
                break
            edges.add((min(a, b), max(a, b)))
        if ok:
            return sorted(edges)
    raise RuntimeError("could not draw a simple regular graph")


def qaoa_params(p: int, seed: int):
    rng = SplitMix64(seed ^ 0x51A0A)
    gammas = [rng.unit() * math.pi for _ in range(p)]
    betas = [rng.unit() * (math.pi / 2.0) for _ in range(p)]
    return gammas, betas


def qaoa_maxcut(n: int, p: int, seed: int) -> Circuit:
    """QAOA MaxCut: ``H^n``, then ``p`` x (RZZ(-gamma_l) on every edge; RX(2 beta_l) on every qubit)."""
    edges = regular_graph(n, seed)
    gammas, betas = qaoa_params(p, seed)
    c = Circuit(n)
    for q in range(n):
        c.h(q)
    for gam, bet in zip(gammas, betas):
        for a, b in edges:
            c.rzz(a, b, -gam)
        for q in range(n):
            c.rx(q, 2.0 * bet)
    return c


def ansatz_circuit(n: int, depth: int, rng: SplitMix64) -> Circuit:
    c = Circuit(n)
    for _ in range(depth):
        for q in range(n):
            theta = rng.angle()
            phi = rng.angle()
            c.rz(q, phi)
            c.ry(q, theta)
        for i in range(n - 1):
            c.cx(i, i + 1)
    return c


def ansatz_batch(count: int, seed: int, n_lo: int = 10, n_hi: int = 20,
                 d_lo: int = 4, d_hi: int = 12) -> list:
    """``count`` layered RY/RZ + CX-ladder circuits with n ~ U{n_lo..n_hi}, depth ~ U{d_lo..d_hi}."""
    rng = SplitMix64(seed)
    out = []
    for _ in range(count):
        n = n_lo + rng.below(n_hi - n_lo + 1)
        d = d_lo + rng.below(d_hi - d_lo + 1)
        out.append(ansatz_circuit(n, d, rng))
    return out
