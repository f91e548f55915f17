"""One state of n qubits spread over 2^g ranks (one GPU each, one process per GPU).

Rank r holds the 2^(n-g) amplitudes whose top g physical index bits equal r ("global" qubits);
the low n-g physical bits are the rank's local qubits, a state the single-GPU engine runs as it
is. The reference keeps a whole state on one device and lists the split across devices as future
work (docs/todo.md:188-191); the index math is the reference's (state/layout.rs:22-86) with the
rank supplying the high bits.

Physical positions are not fixed per logical qubit: a map ``phys[q]`` moves as the circuit runs.

* A gate on local qubits runs on every rank through the engine (``qsvb_execute``: fusion,
  tile sweeps, tensor cores), its qubits renamed to their physical positions.
* A gate whose matrix does not mix the values of its global qubits (diagonals such as CZ, RZZ and
  controlled phases; any gate whose global qubits only act as controls) runs locally too: each
  rank applies the block its own global bits select (for all-global qubits, a phase or nothing).
* Any other gate first brings its global qubits in: an exchange swaps k global positions with the
  k highest local positions. For those, the amplitudes a rank sends to one partner form one
  contiguous block (the local indices whose top k bits take one value), so blocks travel as they
  lie in HBM, with no packing pass. Partners follow an XOR schedule (step s pairs ranks whose
  exchanged bits differ by s), so every step is a set of disjoint pairwise swaps and no rank waits
  on one that is busy elsewhere. A qubit of the gate that sits in that top region moves down first
  by a local SWAP. The local qubits that leave are either those whose next use lies furthest ahead
  (moved into the top positions by local SWAPs) or those already there; the planner keeps the
  choice with less estimated data movement (``plan_cost``).

The exchange goes through a communicator: ``TorchComm`` (torch.distributed; NCCL over
NVLink/NVSwitch between GPUs, gloo on CPU) or none when one process owns every rank (the ranks are
then slices on one device and blocks swap by device copies). The local engine is a
``B200SliceEngine`` over the CUDA library; it is an interface, so the host logic can be tested
with another engine on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from . import gate as G
from .circuit import Circuit
from .gate import DenseGate


# ---------------------------------------------------------------------------------------- plan

@dataclass
class LocalOp:
    """A gate in physical positions. ``glob`` lists (gate bit j, global bit index) of qubits that
    stay global: each rank applies the block its own bits select. ``moved``: a SWAP the planner
    inserted to bring a leaving qubit into the top positions."""
    matrix: np.ndarray
    local: tuple            # (gate bit j, physical position) of the local qubits
    glob: tuple = ()
    moved: bool = False


@dataclass
class LocalStep:
    ops: list = field(default_factory=list)


@dataclass
class ExchangeStep:
    """Swap global bit ``gbits[i]`` with local position ``tpos[i]`` (the top len(tpos) local
    positions, in any order)."""
    gbits: tuple
    tpos: tuple


def _mixes(matrix: np.ndarray, j: int) -> bool:
    """True when the gate has a non-zero element between indices that differ in bit j (exact-zero
    test, the rule of gate.rs:56-68 applied per bit)."""
    d = matrix.shape[0]
    idx = np.arange(d)
    differ = ((idx[:, None] ^ idx[None, :]) >> j) & 1
    return bool(np.any((matrix != 0) & (differ == 1)))


def _next_uses(circuit: Circuit):
    """next_use[i][q]: index of the first gate after gate i that acts on q (or infinity)."""
    ops = circuit.ops()
    n = circuit.n_qubits()
    inf = len(ops) + 1
    nxt = [inf] * n
    out = [None] * len(ops)
    for i in range(len(ops) - 1, -1, -1):
        out[i] = list(nxt)
        for q in ops[i].qubits:
            nxt[q] = i
    return out


def _next_mixing_uses(circuit: Circuit):
    """next_mix[i][q]: index of the first gate after gate i whose matrix mixes q's values (or
    infinity): the next gate that would need q local."""
    ops = circuit.ops()
    n = circuit.n_qubits()
    inf = len(ops) + 1
    nxt = [inf] * n
    out = [None] * len(ops)
    for i in range(len(ops) - 1, -1, -1):
        out[i] = list(nxt)
        for j, q in enumerate(ops[i].qubits):
            if _mixes(ops[i].gate.matrix, j):
                nxt[q] = i
    return out


class Layout:
    """Logical qubit -> physical position (positions >= n_local are global bits)."""

    def __init__(self, n: int, g: int):
        self.n, self.g, self.nl = n, g, n - g
        self.phys = list(range(n))
        self.log = list(range(n))

    def copy(self) -> "Layout":
        c = Layout(self.n, self.g)
        c.phys, c.log = list(self.phys), list(self.log)
        return c

    def swap_positions(self, a: int, b: int):
        qa, qb = self.log[a], self.log[b]
        self.log[a], self.log[b] = qb, qa
        self.phys[qa], self.phys[qb] = b, a

    def physical_index(self, logical_index: int) -> int:
        out = 0
        for q in range(self.n):
            out |= ((logical_index >> q) & 1) << self.phys[q]
        return out


# An exchange moving a whole slice over NVLink (about 770 GB/s per direction) costs this many local
# sweeps (one read and one write of the slice in HBM, about 6.5 TB/s).
EXCHANGE_SWEEPS_PER_SLICE = 6.5e12 / (2 * 770e9)


def plan_cost(steps) -> float:
    """Estimated data movement of a plan beyond its gates, in local sweeps: every exchange of k bits
    moves (1 - 2^-k) of the slice, every planner-inserted SWAP is one local sweep."""
    ex = sum(1.0 - 2.0 ** -len(s.gbits) for s in steps if isinstance(s, ExchangeStep))
    moved = sum(1 for s in steps if isinstance(s, LocalStep) for op in s.ops if op.moved)
    return ex * EXCHANGE_SWEEPS_PER_SLICE + moved


MAX_EXCHANGE_BITS = 4  # global qubits one exchange brings in when it groups upcoming needs


def plan_distributed(circuit: Circuit, g: int, layout: Layout | None = None, policy: str = "auto",
                     group: bool = False):
    """Steps (``LocalStep`` / ``ExchangeStep``) that run ``circuit`` on 2^g ranks from ``layout``
    (identity when None); returns ``(steps, final_layout)``. Every rank computes the same plan.

    ``policy`` picks the local qubits that leave at an exchange: "furthest" (next use furthest
    ahead, moved into the top positions by local SWAPs: fewer exchanges), "top" (whatever sits in
    the top positions, no SWAPs unless a qubit of the gate is there), or "auto" (every policy, with
    and without grouping, keeping the plan with the lowest ``plan_cost``). ``group``: an exchange
    also brings in the global qubits that a gate within the next n gates will need local (k bits
    at once move 1 - 2^-k of the slice, against k/2 one at a time), up to MAX_EXCHANGE_BITS."""
    if policy == "auto":
        plans = [plan_distributed(circuit, g, layout, p, grp) for p in ("furthest", "top") for grp in (False, True)]
        return min(plans, key=lambda pl: plan_cost(pl[0]))
    if policy not in ("furthest", "top"):
        raise ValueError(f"unknown policy {policy!r}")
    n = circuit.n_qubits()
    if g < 0 or n - g < 6:
        raise ValueError("a distributed state needs at least 6 local qubits per rank")
    lay = layout.copy() if layout is not None else Layout(n, g)
    nl = lay.nl
    steps: list = []
    cur = LocalStep()
    nxt = _next_uses(circuit)
    nxm = _next_mixing_uses(circuit) if group else None

    def push_swap(a: int, b: int):
        cur.ops.append(LocalOp(G.swap().matrix, ((0, a), (1, b)), moved=True))
        lay.swap_positions(a, b)

    for i, op in enumerate(circuit.ops()):
        qs, mat = op.qubits, op.gate.matrix
        need = [j for j, q in enumerate(qs) if lay.phys[q] >= nl and _mixes(mat, j)]
        if need:
            gate_q = set(qs)
            # local qubits that may leave: not in this gate
            cand = [q for q in range(n) if lay.phys[q] < nl and q not in gate_q]
            bring = [qs[j] for j in need]
            if group:  # global qubits soon needed local come in with this exchange
                room = min(MAX_EXCHANGE_BITS, len(cand)) - len(bring)
                soon = [q for q in range(n) if lay.phys[q] >= nl and q not in gate_q and nxm[i][q] <= i + n]
                soon.sort(key=lambda q: nxm[i][q])
                bring += soon[:max(0, room)]
            k = len(bring)
            top = list(range(nl - 1, nl - 1 - k, -1))
            if policy == "top":
                cand.sort(key=lambda q: (-lay.phys[q], -nxt[i][q]))
            else:
                cand.sort(key=lambda q: (-nxt[i][q], -lay.phys[q]))
            leave = cand[:k]
            # move the leaving qubits into the top positions (local SWAPs), keeping those already there
            at_top = [q for q in leave if lay.phys[q] in top]
            free_top = [t for t in top if lay.log[t] not in at_top]
            for q in leave:
                if lay.phys[q] not in top:
                    push_swap(lay.phys[q], free_top.pop(0))
            if cur.ops:
                steps.append(cur)
                cur = LocalStep()
            gbits = tuple(lay.phys[q] - nl for q in bring)
            tpos = tuple(lay.phys[q] for q in leave)
            steps.append(ExchangeStep(gbits, tpos))
            for gb, t in zip(gbits, tpos):
                lay.swap_positions(nl + gb, t)
        local = tuple((j, lay.phys[q]) for j, q in enumerate(qs) if lay.phys[q] < nl)
        glob = tuple((j, lay.phys[q] - nl) for j, q in enumerate(qs) if lay.phys[q] >= nl)
        cur.ops.append(LocalOp(mat, local, glob))
    if cur.ops:
        steps.append(cur)
    return steps, lay


def rank_circuit(step: LocalStep, n_local: int, rank: int) -> Circuit:
    """The circuit rank ``rank`` runs for a local step (global qubits fixed to its bits)."""
    c = Circuit(n_local)
    for op in step.ops:
        if not op.glob:
            pos = [p for _, p in op.local]
            c.push(DenseGate(len(pos), op.matrix), pos)
            continue
        fixed = 0
        for j, gb in op.glob:
            fixed |= ((rank >> gb) & 1) << j
        m = len(op.local)
        sub = np.arange(1 << m)
        full = np.full(1 << m, fixed)
        for i, (j, _) in enumerate(op.local):
            full |= ((sub >> i) & 1) << j
        blk = op.matrix[np.ix_(full, full)]
        if np.array_equal(blk, np.eye(1 << m)):
            continue
        if m == 0:  # all qubits global: one phase for the whole slice
            c.push(DenseGate(1, np.eye(2) * blk[0, 0]), [0])
        else:
            c.push(DenseGate(m, blk), [p for _, p in op.local])
    return c


# ------------------------------------------------------------------------------ engines / comms

class _CudaArray:
    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


class B200SliceEngine:
    """The CUDA engine as the per-rank local state: one ``qsvb`` context on this rank's device."""

    def __init__(self, backend):
        import torch
        self.backend = backend
        self.torch = torch
        self.device = torch.device("cuda", torch.cuda.current_device())
        self._stream = torch.cuda.ExternalStream(backend.stream(), device=self.device)

    def alloc(self, n_local: int):
        return self.backend.alloc(n_local)

    def views(self, st):
        """(re, im) torch tensors on the device sharing the state's memory."""
        n = C.c_uint32()
        dt = C.c_int()
        re, im = C.c_void_p(), C.c_void_p()
        L.check(L.lib().qsvb_state_info(st.handle, C.byref(n), C.byref(dt), C.byref(re), C.byref(im)))
        ts = "<f8" if dt.value == L.C128 else "<f4"
        size = 1 << n.value
        mk = lambda p: self.torch.as_tensor(_CudaArray(p.value, size, ts), device=self.device)
        return mk(re), mk(im)

    def stream(self):
        """Context under which torch work (copies, NCCL) queues behind the engine's kernels."""
        return self.torch.cuda.stream(self._stream)

    def init_basis(self, st, basis):
        if basis is None:
            re, im = self.views(st)
            with self.stream():
                re.zero_()
                im.zero_()
        else:
            self.backend.init_basis(st, basis)

    def run(self, st, circuit):
        if len(circuit):
            self.backend.run(st, circuit)

    def expectation_z(self, st, mask: int) -> float:
        return self.backend.expectation_z(st, mask)

    def download(self, st):
        sv = self.backend.download(st)
        return sv.re, sv.im

    def synchronize(self):
        self.backend.synchronize()


class TorchComm:
    """Pairwise block exchange and reductions over torch.distributed (NCCL on GPUs, gloo on CPU).
    Rank i of the process group holds global rank i of the state."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch, self.group = dist, torch, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        if device is None:  # NCCL reduces device tensors only
            nccl = dist.get_backend(group) == "nccl"
            device = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")
        self.device = device

    def exchange(self, send, recv, peer: int):
        """Send the tensors ``send`` to ``peer`` and receive the same shapes into ``recv``."""
        d = self.dist
        ops = [d.P2POp(d.isend, t, peer, self.group) for t in send]
        ops += [d.P2POp(d.irecv, t, peer, self.group) for t in recv]
        for w in d.batch_isend_irecv(ops):
            w.wait()

    def all_reduce(self, values):
        t = self.torch.tensor(values, dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, group=self.group)
        return t.cpu().tolist()

    def gather(self, obj, root: int = 0):
        out = [None] * self.size if self.rank == root else None
        self.dist.gather_object(obj, out, dst=root, group=self.group)
        return out


# ----------------------------------------------------------------------------------- the state

class DistributedState:
    """A state of ``n_qubits`` over ``2**global_qubits`` ranks. ``comm`` None: this process owns
    every rank (slices on one device); otherwise it owns rank ``comm.rank`` and the group has
    ``2**global_qubits`` members. ``chunk_elems``: amplitudes per transfer (the receive buffer).
    ``policy``: the exchange planner's policy (see ``plan_distributed``; "furthest+group" or
    "top+group" for a fixed policy with grouped exchanges)."""

    def __init__(self, n_qubits: int, global_qubits: int, engine, comm=None, chunk_elems: int = 1 << 25,
                 policy: str = "auto"):
        self.n, self.g = int(n_qubits), int(global_qubits)
        self.nl = self.n - self.g
        if self.nl < 6:
            raise ValueError("a distributed state needs at least 6 local qubits per rank")
        self.world = 1 << self.g
        if comm is not None and comm.size != self.world:
            raise ValueError(f"the group has {comm.size} ranks; 2^{self.g} = {self.world} are needed")
        self.engine, self.comm = engine, comm
        self.owned = [comm.rank] if comm is not None else list(range(self.world))
        self.slices = {r: engine.alloc(self.nl) for r in self.owned}
        self.layout = Layout(self.n, self.g)
        self.chunk = max(1, int(chunk_elems))
        self.policy = policy
        self.stats = {"exchanges": 0, "exchanged_bytes_per_rank": 0, "local_steps": 0}

    # -- preparation
    def init_basis(self, basis: int = 0):
        """|basis> in logical order; the layout returns to identity."""
        self.layout = Layout(self.n, self.g)
        p = self.layout.physical_index(int(basis))
        owner, local = p >> self.nl, p & ((1 << self.nl) - 1)
        for r, st in self.slices.items():
            self.engine.init_basis(st, local if r == owner else None)

    # -- circuit
    def run(self, circuit: Circuit) -> dict:
        if circuit.n_qubits() != self.n:
            raise ValueError("circuit width does not match the state")
        policy, grp = self.policy, False
        if policy.endswith("+group"):  # e.g. "top+group": that policy with grouped exchanges
            policy, grp = policy[: -len("+group")], True
        steps, self.layout = plan_distributed(circuit, self.g, self.layout, policy, grp)
        for s in steps:
            if isinstance(s, LocalStep):
                self.stats["local_steps"] += 1
                for r, st in self.slices.items():
                    self.engine.run(st, rank_circuit(s, self.nl, r))
            else:
                self._exchange(s)
        return dict(self.stats)

    def _exchange(self, s: ExchangeStep):
        k = len(s.gbits)
        blk = 1 << (self.nl - k)

        def bits_of(r):  # this rank's exchanged global bits as a k-bit value
            return sum(((r >> gb) & 1) << i for i, gb in enumerate(s.gbits))

        def with_bits(r, v):
            for i, gb in enumerate(s.gbits):
                r = (r & ~(1 << gb)) | (((v >> i) & 1) << gb)
            return r

        def base(v):  # first local index whose top-k bits (tpos) take value v
            return sum(((v >> i) & 1) << t for i, t in enumerate(s.tpos))

        views = {r: self.engine.views(st) for r, st in self.slices.items()}
        tmp = None  # receive buffers, allocated on the first remote transfer
        with self.engine.stream():
            for step in range(1, 1 << k):
                for r in self.owned:
                    a = bits_of(r)
                    v = a ^ step
                    peer = with_bits(r, v)
                    mine = [t[base(v):base(v) + blk] for t in views[r]]
                    if peer in views:  # both slices here: swap block v of r with block a of peer once
                        if r < peer:
                            theirs = [t[base(a):base(a) + blk] for t in views[peer]]
                            for x, y in zip(mine, theirs):
                                for o in range(0, blk, self.chunk):
                                    xa, ya = x[o:o + self.chunk], y[o:o + self.chunk]
                                    tmp = xa.clone()
                                    xa.copy_(ya)
                                    ya.copy_(tmp)
                        continue
                    if tmp is None:
                        tmp = [x.new_empty(min(self.chunk, blk)) for x in mine]
                    for o in range(0, blk, self.chunk):
                        w = min(self.chunk, blk - o)
                        send = [x[o:o + w] for x in mine]
                        recv = [t[:w] for t in tmp]
                        self.comm.exchange(send, recv, peer)
                        for x, t in zip(send, recv):
                            x.copy_(t)
                    self.stats["exchanged_bytes_per_rank"] += 2 * blk * mine[0].element_size()
        self.stats["exchanges"] += 1

    # -- read-out
    def _reduce(self, vals):
        return self.comm.all_reduce(vals) if self.comm is not None else vals

    def expectation_z(self, mask: int) -> float:
        """<Z...Z> over the logical qubits in ``mask`` (sample.rs:177-200), summed over ranks."""
        pm = self.layout.physical_index(int(mask))
        lm, gm = pm & ((1 << self.nl) - 1), pm >> self.nl
        tot = 0.0
        for r, st in self.slices.items():
            sign = -1.0 if bin(r & gm).count("1") & 1 else 1.0
            tot += sign * self.engine.expectation_z(st, lm)
        return self._reduce([tot])[0]

    def norm_sqr(self) -> float:
        return self.expectation_z(0)

    def gather(self, root: int = 0):
        """The whole state in logical index order as complex128 on ``root`` (None elsewhere); for
        states that fit one host."""
        parts = {r: self.engine.download(st) for r, st in self.slices.items()}
        if self.comm is not None:
            got = self.comm.gather((self.comm.rank, parts[self.comm.rank]), root)
            if self.comm.rank != root:
                return None
            parts = dict(got)
        phys = np.concatenate([np.asarray(parts[r][0], np.float64) + 1j * np.asarray(parts[r][1], np.float64)
                               for r in range(self.world)])
        # physical index bit p holds logical qubit log[p]: reorder axes to logical order
        t = phys.reshape((2,) * self.n)             # axis a <-> physical bit n-1-a
        axes = [self.n - 1 - self.layout.phys[self.n - 1 - a] for a in range(self.n)]
        return np.ascontiguousarray(t.transpose(axes)).reshape(-1)

    def free(self):
        for st in self.slices.values():
            if hasattr(st, "free"):
                st.free()
        self.slices = {}
