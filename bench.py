"""Benchmark: 30-qubit random brickwork circuit (complex64, depth 20) on one B200.

Metric (lower is better): circuit seconds of the tensor-core + learned-fusion plan, with the
plain GPU paths (unfused, greedy-fused on CUDA cores at k=2..6) measured beside it and the
infidelity 1-F of the result against an FP64 (complex128) run of the same circuit.

A step = one execution of the circuit from |0..0> (init + every sweep) on a resident 8 GiB state
(larger than L2, so no flush is needed). Timing: CUDA events on the engine's stream, W warm-up
steps, K timed steps bracketed by barrier + synchronize, max over ranks. With N GPUs every rank
runs its own replica of the circuit (the single-state path does not shard): value stays the
circuit time (the max over ranks of the step time), and the whole job's throughput is reported
separately as circuits_per_second = N / value.

``--impl reference`` times the CPU restatement of qsv's CpuBackend (OpenMP over all host cores)
on a bounded sample of the same workload and extrapolates to the full circuit.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "30q circuit sec: TC+learned fusion vs plain GPU at 1-F<=1e-5; HBM GB/s/peak"
N_QUBITS, DEPTH, SEED = 30, 20, 0
WORKLOAD = f"random brickwork {N_QUBITS}q depth {DEPTH}, complex64, Haar SU(2) + CZ, seed {SEED}"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum, one ncu capture of one launch at 26
# qubits, scaled by the amplitudes a launch processes) per algorithmic byte, for the kernels the
# roofline object can name
TRAFFIC_PER_ALGORITHMIC_BYTE = {"dense_tc": (537.161472 + 476.718592) / 1073.741824,
                                "tc_chain": (537.134848 + 477.886720) / 1073.741824,
                                "1q": (536.916992 + 479.222272) / 1073.741824}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks sampling
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline (oracle CpuBackend)
def cpu_baseline(circuit, budget_s: float = 15.0) -> dict:
    """Time the CpuBackend restatement (OpenMP, all host threads) on the reference-fused circuit
    (FusionConfig default max_qubits=4, composed in f32 as qsv does for Circuit<f32>). Ops are
    sampled round-robin over their arities (a seeded order within each arity) until the time budget
    is spent; the estimate is sum over arities of (ops of that arity) x (mean time of the sampled
    ones), so it does not depend on which ops come first in the circuit."""
    import oracle
    n = circuit.n_qubits()
    arity, qubits, mats = oracle.fuse(circuit, 4, oracle.F32)
    nops = len(arity)
    L = oracle.lib()
    cores = int(L.orc_max_threads())
    re = np.zeros(1 << n, dtype=np.float32)
    im = np.zeros(1 << n, dtype=np.float32)
    re[0] = 1.0
    offs_q = np.concatenate([[0], np.cumsum(arity)]).astype(np.int64)
    offs_m = np.concatenate([[0], np.cumsum([2 * (1 << (2 * int(m))) for m in arity])]).astype(np.int64)

    def run_op(i):
        m = int(arity[i])
        L.orc_apply(oracle.CPU_PARALLEL, oracle.F32, n, re.ctypes.data, im.ctypes.data,
                    np.ascontiguousarray(mats[offs_m[i]:offs_m[i + 1]]),
                    np.ascontiguousarray(qubits[offs_q[i]:offs_q[i + 1]]), m)

    rng = np.random.default_rng(SEED)
    classes = {}
    for i in rng.permutation(nops):
        classes.setdefault(int(arity[i]), []).append(int(i))
    order = []
    for r in range(max(len(v) for v in classes.values())):
        for m in sorted(classes):
            if r < len(classes[m]):
                order.append(classes[m][r])
    run_op(order[0])  # first touch of the pages, untimed
    times = {m: [] for m in classes}
    t0 = time.perf_counter()
    for i in order:
        t = time.perf_counter()
        run_op(i)
        times[int(arity[i])].append(time.perf_counter() - t)
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    done = sum(len(v) for v in times.values())
    mean_all = dt / max(done, 1)
    est = sum(len(classes[m]) * (float(np.mean(times[m])) if times[m] else mean_all) for m in classes)
    hist = ", ".join(f"{len(times[m])}/{len(classes[m])} of arity {m}" for m in sorted(classes))
    return {"value": est, "unit": "s", "cores": cores, "kind": "port",
            "sample": f"{done} of {nops} fused ops (qsv fuse, max_qubits=4, f32) of the {n}q circuit timed "
                      f"({hist}; {dt:.1f} s, OpenMP x{cores}); value = sum over arities of ops x mean time"}


def lscpu_summary() -> dict:
    """Host CPU facts for the baseline (lscpu), so the core count the baseline uses is checkable."""
    keys = ("Model name", "Socket(s)", "Core(s) per socket", "Thread(s) per core", "CPU(s)", "NUMA node(s)")
    out = {}
    try:
        txt = subprocess.run(["lscpu"], capture_output=True, text=True, timeout=10).stdout
        for line in txt.splitlines():
            k, _, v = line.partition(":")
            if k.strip() in keys:
                out[k.strip()] = v.strip()
    except Exception as e:  # lscpu missing: report why
        out["error"] = str(e)
    return out


def cpu_full_circuits(sizes=(24, 26, 28)) -> dict:
    """The CpuBackend restatement (OpenMP, all host threads) on the WHOLE reference-fused brickwork
    circuit (same depth and seed) at smaller sizes: every op timed, nothing sampled. These anchor
    the sampled 30-qubit estimate; the per-amplitude cost at 28 qubits times 4 is a second,
    fully-timed extrapolation to 30 qubits."""
    import oracle
    from rustatevec_b200.circuits import brickwork
    L = oracle.lib()
    out = {}
    for n in sizes:
        c = brickwork(n, DEPTH, SEED)
        arity, qubits, mats = oracle.fuse(c, 4, oracle.F32)
        re = np.zeros(1 << n, dtype=np.float32)
        im = np.zeros(1 << n, dtype=np.float32)
        re[0] = 1.0
        t0 = time.perf_counter()
        rc = L.orc_run(oracle.CPU_PARALLEL, oracle.F32, n, re.ctypes.data, im.ctypes.data, len(arity), arity, qubits,
                       mats)
        out[str(n)] = round(time.perf_counter() - t0, 3)
        if rc:
            raise RuntimeError("oracle rejected the circuit")
    if "28" in out:
        out["extrapolated_30q_from_28q"] = round(out["28"] * 4.0, 2)
    return out


# ------------------------------------------------------------------ GPU
def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    return world, rank, local


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def run_gpu(args):
    import torch
    from rustatevec_b200 import (B200Backend, Plan, PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_LEARNED, PLAN_WINDOW,
                                 ENGINE_AUTO, ENGINE_CUDA_CORE, ENGINE_TENSOR_CORE)
    from rustatevec_b200 import _lib as L
    from rustatevec_b200.circuits import brickwork

    from rustatevec_b200 import tuning
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    model_doc = tuning.load()  # the learned cost model trained on B200 measurements (None: roofline model)
    be = B200Backend(local, precision="f32")
    stream = torch.cuda.ExternalStream(be.stream(), device=torch.device("cuda", local))
    circuit = brickwork(N_QUBITS, DEPTH, SEED)
    state = be.alloc(N_QUBITS)

    def timed(plan, steps, warmup):
        for _ in range(warmup):
            be.init_basis(state, 0)
            plan.run(state)
        be.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            be.init_basis(state, 0)
            plan.run(state)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        barrier(world)
        return e0.elapsed_time(e1) * 1e-3 / steps

    methods = {
        "unfused": L.make_opts(PLAN_AS_GIVEN, 1, ENGINE_CUDA_CORE),
        **{f"greedy_k{k}_cuda": L.make_opts(PLAN_GREEDY, k, ENGINE_CUDA_CORE) for k in (2, 3, 4, 5, 6)},
        "window_k4_cuda": L.make_opts(PLAN_WINDOW, 4, ENGINE_CUDA_CORE),
        "learned_cuda": L.make_opts(PLAN_LEARNED, 6, ENGINE_CUDA_CORE),
        "greedy_k6_tc": L.make_opts(PLAN_GREEDY, 6, ENGINE_TENSOR_CORE),
        "window_k6_tc": L.make_opts(PLAN_WINDOW, 6, ENGINE_TENSOR_CORE),
        "tile": L.make_opts(L.PLAN_TILE, 4, ENGINE_AUTO),
        "chain_m2": L.make_opts(L.PLAN_CHAIN, 6, ENGINE_AUTO, chain_max_matrices=2),
        "chain_m3": L.make_opts(L.PLAN_CHAIN, 6, ENGINE_AUTO, chain_max_matrices=3),
        # the learned planner with the cost model removed (its analytic roofline model instead)
        "learned_tc_roofline_model": L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO),
        "learned_tc": L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO),
    }
    headline = "learned_tc"
    results = {}
    plans = {}
    for name, o in methods.items():
        if name == "learned_tc_roofline_model":
            tuning.install(None)
            p = Plan(be, circuit, o)
            if model_doc:
                tuning.install(model_doc["model"])
        else:
            p = Plan(be, circuit, o)
        plans[name] = p
        if name == headline or args.quick:
            continue
        t = timed(p, steps=2, warmup=1)
        st = p.stats()
        results[name] = {"seconds": allreduce_max(t, world), "sweeps": st["n_sweeps"], "by_kind": st["by_kind"]}

    hp = plans[headline]
    clocks = ClockSampler(local)
    clocks.start()
    t_step = timed(hp, args.steps, args.warmup)
    clk = clocks.stop()
    t_step = allreduce_max(t_step, world)
    hst = hp.stats()
    results[headline] = {"seconds": t_step, "sweeps": hst["n_sweeps"], "by_kind": hst["by_kind"]}

    out = None
    if rank == 0:
        # the plain GPU method of the configuration: qsv's fuse at max k = 2..6 (or no fusion), every
        # sweep on CUDA cores; the engine's other CUDA-core plans (window, learned, tile) beside it
        plain = {k: v["seconds"] for k, v in results.items() if k.startswith("greedy_k") and k.endswith("_cuda")
                 or k == "unfused"}
        best_plain = min(plain.items(), key=lambda kv: kv[1]) if plain else (None, None)
        cuda_any = {k: v["seconds"] for k, v in results.items() if k.endswith("_cuda") or k in ("unfused", "tile")}
        best_cuda_any = min(cuda_any.items(), key=lambda kv: kv[1]) if cuda_any else (None, None)

        # fidelity of the headline state against an FP64 run of the same circuit
        be.init_basis(state, 0)
        hp.run(state)
        be64 = B200Backend(local, precision="f64")
        s64 = be64.alloc(N_QUBITS)
        be64.init_basis(s64, 0)
        be64.run(s64, circuit, L.make_opts(PLAN_GREEDY, 4, ENGINE_CUDA_CORE))
        be64.synchronize()
        ip = np.zeros(2)
        import ctypes as C
        L.check(L.lib().qsvb_inner_product(be.ctx, state.handle, s64.handle, ip.ctypes.data_as(L._dp)))
        n32 = be.norm_sqr(state)
        fid = (ip[0] ** 2 + ip[1] ** 2) / n32
        s64.free()
        be64.close()

        # roofline of the dominant kernel: per-sweep device times of the headline plan
        sweeps = hp.sweeps()
        per = hp.profile(state, reps=2)
        by_kind = {}
        for s, t in zip(sweeps, per):
            d = by_kind.setdefault(s["kind"], {"time": 0.0, "bytes": 0.0, "flops": 0.0, "launches": 0})
            d["time"] += t
            d["bytes"] += s["algorithmic_bytes"]
            d["flops"] += s["flops"]
            d["launches"] += 1
        dom = max(by_kind, key=lambda k: by_kind[k]["time"])
        d = by_kind[dom]
        peak, peak_kind = peaks()
        achieved = d["bytes"] / d["time"] / 1e9
        ratio = TRAFFIC_PER_ALGORITHMIC_BYTE.get(dom)
        roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "traffic": round(ratio * d["bytes"] / d["launches"]) if ratio else None,
                    "traffic_source": "ncu dram bytes of one launch at 26 qubits, scaled by amplitudes" if ratio else None,
                    "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                    "avg_launch_us": round(d["time"] / d["launches"] * 1e6, 1),
                    "algorithmic_bytes_per_launch": d["bytes"] / d["launches"],
                    "share_of_step": round(d["time"] / max(sum(v["time"] for v in by_kind.values()), 1e-30), 3),
                    "by_kind": {k: {"launches": v["launches"], "seconds": round(v["time"], 5),
                                    "GB/s": round(v["bytes"] / v["time"] / 1e9, 1) if v["time"] else None}
                                for k, v in by_kind.items()}}

        # end to end through the public API: host circuit -> execute -> <Z_0> back on the host
        e2e_steps = max(2, min(args.steps, 4))
        pc_bytes = sum(2 * 8 * (1 << (2 * len(op.qubits))) for op in circuit.ops())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        be.synchronize()
        e0.record(stream)
        for _ in range(e2e_steps):
            be.init_basis(state, 0)
            be.run(state, circuit, methods[headline])
            _ = be.expectation_z(state, 1)
        e1.record(stream)
        e1.synchronize()
        e2e = e0.elapsed_time(e1) * 1e-3 / e2e_steps

        cpu = cpu_baseline(circuit, budget_s=args.cpu_budget) if not args.no_cpu else None
        if cpu is not None:
            cpu["lscpu"] = lscpu_summary()
            if not args.no_cpu_scaling:
                cpu["full_circuit_seconds"] = cpu_full_circuits()
        n_launch = args.steps * (hst["n_sweeps"] + 1)
        out = {
            "metric": METRIC, "value": round(t_step, 6), "unit": "s", "n_gpus": world,
            "circuits_per_second": round(world / t_step, 3),
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_step * 1e3, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 state (complex64); k>=5 dense sweeps on tcgen05 bf16 hi/lo, fp32 accumulate",
            "data": "synthetic (seeded brickwork circuit)",
            "config": {"workload": WORKLOAD, "n_qubits": N_QUBITS, "depth": DEPTH, "gates": len(circuit),
                       "plan": headline, "plan_sweeps": hst["n_sweeps"], "plan_by_kind": hst["by_kind"],
                       "l2": "state is 8 GiB (> 126 MB L2): no flush needed",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "infidelity_vs_fp64": float(1.0 - fid),
            "cost_model": (model_doc or {}).get("meta", "none (roofline model)"),
            "methods_seconds": {k: round(v["seconds"], 5) for k, v in results.items()},
            "methods_sweeps": {k: v["sweeps"] for k, v in results.items()},
            "best_plain_gpu": {"method": best_plain[0], "seconds": best_plain[1],
                               "definition": "qsv fuse (greedy) at max k=2..6 or unfused, CUDA cores",
                               "speedup_of_headline": (best_plain[1] / t_step) if best_plain[1] else None},
            "best_cuda_core_any": {"method": best_cuda_any[0], "seconds": best_cuda_any[1],
                                   "speedup_of_headline": (best_cuda_any[1] / t_step) if best_cuda_any[1] else None},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e, 6), "unit": "s", "h2d_bytes_per_step": pc_bytes, "d2h_bytes_per_step": 16,
                    "path": "B200Backend.run(host circuit) -> qsvb_execute (plan + matrix upload + sweeps) -> "
                            "expectation_z(mask=1) read back"},
            "gpu_launches": n_launch,
            "clocks": clk,
        }
        print(json.dumps(out), flush=True)
    state.free()
    be.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from rustatevec_b200.circuits import brickwork
    circuit = brickwork(N_QUBITS, DEPTH, SEED)
    vals = []
    last = None
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(circuit, budget_s=args.ref_budget)
        if i >= args.warmup:
            vals.append(r["value"])
        last = r
    v = float(np.mean(vals))
    out = {"impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 (complex64)", "data": "synthetic (seeded brickwork circuit)",
           "config": {"workload": WORKLOAD, "n_qubits": N_QUBITS, "depth": DEPTH},
           "cpu_baseline": {"value": round(v, 3), "unit": "s", "cores": last["cores"], "kind": last["kind"],
                            "sample": last["sample"], "lscpu": lscpu_summary()},
           "e2e": {"value": round(v, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ the other configurations
# Each prints one JSON line with the same keys as the headline (value, roofline, cpu_baseline, e2e,
# clocks, gpu_launches) for its own workload; they are not the default bench line.

def _events(stream):
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def device_seconds(be, stream, body, steps, warmup):
    """Mean device seconds of ``body()`` (which queues work on the engine's stream)."""
    for _ in range(warmup):
        body()
    be.synchronize()
    e0, e1 = _events(stream)
    e0.record(stream)
    for _ in range(steps):
        body()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1) * 1e-3 / steps


def plan_roofline(plan, state, reps=1):
    """Dominant sweep kind of a plan from its per-sweep device times: algorithmic GB/s vs peak."""
    sweeps = plan.sweeps()
    per = plan.profile(state, reps=reps)
    by_kind = {}
    for s, t in zip(sweeps, per):
        d = by_kind.setdefault(s["kind"], {"time": 0.0, "bytes": 0.0, "launches": 0})
        d["time"] += t
        d["bytes"] += s["algorithmic_bytes"]
        d["launches"] += 1
    dom = max(by_kind, key=lambda k: by_kind[k]["time"])
    d = by_kind[dom]
    peak, kind = peaks()
    achieved = d["bytes"] / d["time"] / 1e9
    return {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": None, "peak_source": f"{kind} hbm_gbs",
            "avg_launch_us": round(d["time"] / d["launches"] * 1e6, 1),
            "algorithmic_bytes_per_launch": d["bytes"] / d["launches"],
            "by_kind": {k: {"launches": v["launches"], "seconds": round(v["time"], 5),
                            "GB/s": round(v["bytes"] / v["time"] / 1e9, 1) if v["time"] else None}
                        for k, v in by_kind.items()}}


def _line(metric, value, unit, args, dtype, config, **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": dtype, "data": "synthetic (seeded)", "config": config}
    out.update(extra)
    print(json.dumps(out), flush=True)


def run_config_ghz24(args):
    """GHZ(24) complex128: H(0), CX(i, i+1); all 2^24 FP64 probabilities; p_0 = p_last = 1/2."""
    import torch
    from rustatevec_b200 import B200Backend, Plan, PLAN_AS_GIVEN, PLAN_LEARNED, ENGINE_AUTO, ENGINE_CUDA_CORE
    from rustatevec_b200 import _lib as L
    from rustatevec_b200.circuits import ghz_chain
    from rustatevec_b200 import tuning
    tuning.load()
    n = 24
    circ = ghz_chain(n)
    be = B200Backend(0, precision="f64")
    stream = torch.cuda.ExternalStream(be.stream())
    st = be.alloc(n)
    plans = {"unfused": Plan(be, circ, L.make_opts(PLAN_AS_GIVEN, 1, ENGINE_CUDA_CORE)),
             "tile": Plan(be, circ, L.make_opts(L.PLAN_TILE, 4, ENGINE_AUTO)),
             "learned": Plan(be, circ, L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO))}
    secs = {}
    for name, p in plans.items():
        secs[name] = device_seconds(be, stream, lambda: (be.init_basis(st, 0), p.run(st)), args.steps, args.warmup)
    clocks = ClockSampler(0)
    clocks.start()
    t = device_seconds(be, stream, lambda: (be.init_basis(st, 0), plans["learned"].run(st)), args.steps, args.warmup)
    clk = clocks.stop()
    probs = be.probabilities(st, fp64=True)
    ok = abs(probs[0] - 0.5) < 1e-12 and abs(probs[-1] - 0.5) < 1e-12 and abs(probs.sum() - 1) < 1e-12
    t0 = time.perf_counter()
    for _ in range(args.steps):
        be.init_basis(st, 0)
        be.run(st, circ, L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO))
        probs = be.probabilities(st, fp64=True)
    e2e = (time.perf_counter() - t0) / args.steps
    rl = plan_roofline(plans["learned"], st, reps=3)
    cpu = None
    if not args.no_cpu:
        import oracle
        t0 = time.perf_counter()
        re, im = oracle.run(circ, oracle.CPU_PARALLEL, oracle.F64)
        cpu = {"value": round(time.perf_counter() - t0, 4), "unit": "s", "cores": int(oracle.lib().orc_max_threads()),
               "kind": "port", "sample": "whole circuit (24 gates) on the CpuBackend restatement, FP64"}
    _line("GHZ(24) c128 circuit seconds (graph) + FP64 probabilities", round(t, 7), "s", args, "f64 (complex128)",
          {"workload": "GHZ chain H(0), CX(i,i+1), 24 qubits, complex128", "plan_sweeps":
           plans["learned"].stats()["n_sweeps"], "l2": "256 MiB state (> L2)"},
          methods_seconds={k: round(v, 7) for k, v in secs.items()}, known_answer_ok=bool(ok),
          roofline=rl, cpu_baseline=cpu, clocks=clk, gpu_launches=args.steps * (plans["learned"].stats()["n_sweeps"] + 1),
          e2e={"value": round(e2e, 6), "unit": "s", "h2d_bytes_per_step": sum(32 * (1 << (2 * len(o.qubits))) // 2 for o in circ.ops()),
               "d2h_bytes_per_step": 8 << n, "path": "run(host circuit) + probabilities(fp64) download"})
    st.free()
    be.close()


def run_config_qft32(args):
    """QFT(32) complex64 on an i.i.d. complex Gaussian state: learned vs greedy k=5 vs unfused, with
    the fidelity of each against an FP64 (complex128) run of the same circuit on the same input."""
    import torch
    from rustatevec_b200 import (B200Backend, Plan, PLAN_AS_GIVEN, PLAN_GREEDY, PLAN_LEARNED, ENGINE_AUTO,
                                 ENGINE_CUDA_CORE)
    from rustatevec_b200 import _lib as L
    from rustatevec_b200.circuits import qft
    from rustatevec_b200 import tuning
    tuning.load()
    n = args.qubits if args.qubits != 30 else 32
    seed = SEED
    circ = qft(n)
    be = B200Backend(0, precision="f32")
    stream = torch.cuda.ExternalStream(be.stream())
    st = be.alloc(n)
    methods = {"unfused": L.make_opts(PLAN_AS_GIVEN, 1, ENGINE_CUDA_CORE),
               "greedy_k5": L.make_opts(PLAN_GREEDY, 5, ENGINE_CUDA_CORE),
               "tile": L.make_opts(L.PLAN_TILE, 4, ENGINE_AUTO),
               "learned": L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO)}
    plans = {k: Plan(be, circ, o) for k, o in methods.items()}
    secs = {}
    for name, p in plans.items():
        reps = 1 if name == "unfused" else args.steps
        secs[name] = device_seconds(be, stream, lambda: (be.init_gaussian(st, seed), p.run(st)), reps,
                                    1 if name == "unfused" else args.warmup)
    # FP64 reference state, then the fidelity of every method's result against it
    be64 = B200Backend(0, precision="f64")
    s64 = be64.alloc(n)
    be64.init_gaussian(s64, seed)
    be64.run(s64, circ, L.make_opts(PLAN_GREEDY, 4, ENGINE_CUDA_CORE))
    be64.synchronize()
    fids = {}
    for name, p in plans.items():
        be.init_gaussian(st, seed)
        p.run(st)
        be.synchronize()
        ip = be.inner_product(st, s64)
        fids[name] = float(1.0 - abs(ip) ** 2 / be.norm_sqr(st))
    s64.free()
    be64.close()
    clocks = ClockSampler(0)
    clocks.start()
    t = device_seconds(be, stream, lambda: (be.init_gaussian(st, seed), plans["learned"].run(st)), args.steps,
                       args.warmup)
    clk = clocks.stop()
    rl = plan_roofline(plans["learned"], st)
    t0 = time.perf_counter()
    be.init_gaussian(st, seed)
    be.run(st, circ, methods["learned"])
    z = be.expectation_z(st, 1)
    e2e = time.perf_counter() - t0
    cpu = None
    if not args.no_cpu:
        cpu = cpu_baseline(circ, budget_s=args.cpu_budget)
    _line(f"QFT({n}) c64 circuit seconds on a Gaussian state: learned vs greedy k=5 vs unfused", round(t, 6), "s",
          args, "f32 state (complex64); plan composed in FP64",
          {"workload": f"QFT({n}) complex64, input i.i.d. complex Gaussian (seed {seed}), normalised in FP64",
           "plan_sweeps": {k: p.stats()["n_sweeps"] for k, p in plans.items()}, "l2": "32 GiB state (> L2)"},
          methods_seconds={k: round(v, 5) for k, v in secs.items()}, infidelity_vs_fp64=fids,
          speedup_learned_vs_greedy_k5=round(secs["greedy_k5"] / t, 3),
          speedup_learned_vs_unfused=round(secs["unfused"] / t, 3),
          roofline=rl, cpu_baseline=cpu, clocks=clk, gpu_launches=args.steps * (plans["learned"].stats()["n_sweeps"] + 3),
          e2e={"value": round(e2e, 6), "unit": "s", "h2d_bytes_per_step": sum(16 << (2 * len(o.qubits)) for o in circ.ops()),
               "d2h_bytes_per_step": 8, "path": "init_gaussian + run(host circuit) + expectation_z(mask=1)",
               "z0": z})
    st.free()
    be.close()


def run_config_qaoa33(args):
    """QAOA MaxCut 33 qubits complex128 (137 GB state), p=4: learned vs greedy, FP64 invariants."""
    import torch
    from rustatevec_b200 import B200Backend, Plan, PLAN_GREEDY, PLAN_LEARNED, ENGINE_AUTO, ENGINE_CUDA_CORE
    from rustatevec_b200 import _lib as L
    from rustatevec_b200.circuits import qaoa_maxcut
    from rustatevec_b200 import tuning
    tuning.load()
    n = args.qubits if args.qubits != 30 else 33
    circ = qaoa_maxcut(n, 4, SEED)
    be = B200Backend(0, precision="f64")
    stream = torch.cuda.ExternalStream(be.stream())
    st = be.alloc(n)
    methods = {"greedy_k4": L.make_opts(PLAN_GREEDY, 4, ENGINE_CUDA_CORE),
               "tile": L.make_opts(L.PLAN_TILE, 4, ENGINE_AUTO),
               "learned": L.make_opts(PLAN_LEARNED, 6, ENGINE_AUTO)}
    plans = {k: Plan(be, circ, o) for k, o in methods.items()}
    secs, checks = {}, {}
    masks = [1, 3, 1 << (n - 1), (1 << n) - 1, 0x5555555555555555 & ((1 << n) - 1)]
    for name, p in plans.items():
        secs[name] = device_seconds(be, stream, lambda: (be.init_basis(st, 0), p.run(st)), 1, 1)
        checks[name] = {"norm": be.norm_sqr(st), "z": [be.expectation_z(st, m) for m in masks],
                        "amp": [be.amplitude(st, i) for i in (0, 12345, (1 << n) - 1)]}
    g, l = checks["greedy_k4"], checks["learned"]
    diff = max([abs(a - b) for a, b in zip(g["z"], l["z"])] + [abs(a - b) for a, b in zip(g["amp"], l["amp"])])
    clocks = ClockSampler(0)
    clocks.start()
    t = device_seconds(be, stream, lambda: (be.init_basis(st, 0), plans["learned"].run(st)), max(1, args.steps // 2), 1)
    clk = clocks.stop()
    rl = plan_roofline(plans["learned"], st)
    _line(f"QAOA MaxCut {n}q c128 p=4 circuit seconds: learned vs greedy", round(t, 5), "s", args,
          "f64 (complex128) throughout",
          {"workload": f"QAOA MaxCut {n} qubits, p=4, 3-regular graph (odd n: node 0 degree 4), seed {SEED}",
           "plan_sweeps": {k: p.stats()["n_sweeps"] for k, p in plans.items()},
           "plan_by_kind": {k: p.stats()["by_kind"] for k, p in plans.items()}, "state_GB": 16 * 2 ** n / 1e9},
          methods_seconds={k: round(v, 5) for k, v in secs.items()},
          speedup_learned_vs_greedy=round(secs["greedy_k4"] / t, 3),
          fp64_invariants={"norm_minus_1": {k: v["norm"] - 1.0 for k, v in checks.items()},
                           "max_abs_diff_learned_vs_greedy": diff, "z_masks": masks, "z_learned": l["z"]},
          roofline=rl, cpu_baseline={"value": None, "unit": "s", "cores": None, "kind": "port",
                                     "sample": "not run (RAM): the 137 GB state does not fit the host"},
          clocks=clk, gpu_launches=max(1, args.steps // 2) * (plans["learned"].stats()["n_sweeps"] + 1),
          e2e={"value": None, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
               "note": "device-resident workload; see value"})
    st.free()
    be.close()


def run_config_batched(args):
    """4096 uneven ansatz circuits (n ~ U{10..20}, depth ~ U{4..12}) in one persistent kernel from a
    captured graph, complex64 and complex128, autotuned tiles; <Z_0> + FP64 probabilities per circuit."""
    import ctypes as C
    from rustatevec_b200 import B200Backend
    from rustatevec_b200 import _lib as L
    from rustatevec_b200.circuits import ansatz_batch
    from rustatevec_b200.shard import lpt_partition, circuit_cost
    world, rank, local = dist_setup()
    count = args.circuits
    circuits = ansatz_batch(count, SEED)
    parts = lpt_partition([circuit_cost(c) for c in circuits], world)
    mine = [circuits[i] for i in parts[rank]]
    pb = L.PackedBatch(mine)
    res = {}
    clk = None
    for prec in ("f32", "f64"):
        be = B200Backend(local, precision=prec)
        best_l, best_r = C.c_uint32(0), C.c_uint32(0)
        secs = np.zeros(6)
        cnt = C.c_size_t(0)
        if not args.no_autotune:
            L.check(L.lib().qsvb_batch_autotune(be.ctx, pb.ptr(), pb.count, be.dtype, C.byref(best_l),
                                                C.byref(best_r), secs.ctypes.data_as(L._dp), 6, C.byref(cnt)))
        h = C.c_void_p()
        L.check(L.lib().qsvb_batch_create(be.ctx, pb.ptr(), pb.count, be.dtype, best_l.value, best_r.value,
                                          C.byref(h)))
        z0 = np.zeros(pb.count)
        stt = L.PlanStats()
        for _ in range(args.warmup):
            L.check(L.lib().qsvb_batch_run(be.ctx, h, None, None, None, C.byref(stt)))
        if prec == "f32":
            clocks = ClockSampler(local)
            clocks.start()
        barrier(world)
        ts = []
        for _ in range(args.steps):
            L.check(L.lib().qsvb_batch_run(be.ctx, h, None, None, None, C.byref(stt)))
            ts.append(stt.measured_seconds)
        if prec == "f32":
            clk = clocks.stop()
        t = allreduce_max(float(np.mean(ts)), world)
        # end to end: host circuits -> plan + graph -> run -> <Z_0> and all FP64 probabilities on the host
        t0 = time.perf_counter()
        z0, probs, st2 = be.execute_batch(mine, probabilities=True, local_qubits=best_l.value,
                                          register_qubits=best_r.value)
        e2e = allreduce_max(time.perf_counter() - t0, world)
        d = stt.to_dict()
        L.check(L.lib().qsvb_batch_free(be.ctx, h))
        res[prec] = {"seconds": t, "tile": [best_l.value, best_r.value],
                     "autotune_seconds": [round(x, 5) for x in secs[:cnt.value]],
                     "passes": d["n_sweeps"], "phases": d["by_kind"].get("1q"),
                     "algorithmic_GB": d["algorithmic_bytes"] / 1e9, "flops": d["flops"], "e2e": e2e,
                     "probs_bytes": int(sum(p.nbytes for p in probs)), "z0_sample": [float(x) for x in z0[:3]]}
        be.close()
    if rank != 0:
        return
    peak, kind = peaks()
    r32 = res["f32"]
    ach = r32["algorithmic_GB"] * world / r32["seconds"]
    cpu = None
    if not args.no_cpu:
        import oracle
        rng = np.random.default_rng(0)
        pick = rng.permutation(count)
        t0 = time.perf_counter()
        done_cost = 0.0
        for i in pick:
            c = circuits[int(i)]
            re, im = oracle.run(c, oracle.CPU_PARALLEL, oracle.F32)
            oracle.expectation_z((re.astype(np.float64) ** 2 + im.astype(np.float64) ** 2), 1)
            done_cost += circuit_cost(c)
            if time.perf_counter() - t0 > args.cpu_budget:
                break
        dt = time.perf_counter() - t0
        total = sum(circuit_cost(c) for c in circuits)
        cpu = {"value": round(dt * total / done_cost, 3), "unit": "s", "cores": int(oracle.lib().orc_max_threads()),
               "kind": "port", "sample": f"random circuits of the batch on the CpuBackend restatement (f32) for "
                                         f"{dt:.1f} s, extrapolated by sum(2^n * gates)"}
    _line("batched ansatz: 4096 circuits, seconds per batch (c64; c128 beside)", round(r32["seconds"] / 1.0, 6), "s",
          args, "f32 state (complex64); c128 run beside",
          {"workload": f"{count} ansatz circuits n~U{{10..20}} depth~U{{4..12}} RY.RZ + CX ladder, seed {SEED}",
           "parallelism": f"circuits sharded over {world} GPU(s) by cost (LPT), no collective" if world > 1 else
           "single GPU", "l2": "states and probabilities (6.2 GB) exceed L2"},
          n_gpus=world, by_precision=res, circuits_per_second=round(count / r32["seconds"], 1),
          roofline={"bound": "fp32 (CUDA-core register tiles)", "achieved": round(ach, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(ach / peak, 4), "traffic": None,
                    "achieved_tflops": round(r32["flops"] * world / r32["seconds"] / 1e12, 2),
                    "note": "algorithmic HBM bytes (multi-pass tiles + probabilities) / device time; the kernel "
                            "works out of shared memory and registers, so the HBM fraction is low by design"},
          cpu_baseline=cpu, clocks=clk, gpu_launches=2 * args.steps,
          e2e={"value": round(r32["e2e"], 4), "unit": "s", "h2d_bytes_per_step": None,
               "d2h_bytes_per_step": r32["probs_bytes"] + 8 * count,
               "path": "execute_batch(host circuits): plan + upload + graph run + <Z_0> and probabilities to host"})


KERNEL_CASES = {
    # name: (precision, builder(n) -> circuit with one sweep of that kind, engine)
    "1q_low": ("f32", lambda n: [("h", [1])]),
    "1q_mid": ("f32", lambda n: [("h", [4])]),
    "1q_high": ("f32", lambda n: [("h", [n - 1])]),
    "cx_high": ("f32", lambda n: [("cx", [n - 1, n - 2])]),
    "cz_high": ("f32", lambda n: [("cz", [n - 1, n - 2])]),
    # FP64 reductions (no circuit): <Z_mask> over the whole state, one read of it per call
    "reduce_z": ("f32", lambda n: []),
    "reduce_z_c128": ("f64", lambda n: []),
    "dense4_cuda": ("f32", lambda n: [("u4", [0, 1, 2, 3])]),
    "dense6_cuda": ("f32", lambda n: [("u6", list(range(6)))]),
    "tc4": ("f32", lambda n: [("u4", [0, 1, 2, 3])]),
    "tc6": ("f32", lambda n: [("u6", list(range(6)))]),
    "tc6_high": ("f32", lambda n: [("u6", list(range(n - 6, n)))]),
    "tc6_bit1": ("f32", lambda n: [("u6", [1, 2, 7, 8, 9, 10])]),
    "tc6_bit0": ("f32", lambda n: [("u6", [0, 3, 4, 8, 9, 12])]),
    "phase15": ("f32", lambda n: [("cz", [i, i + 1]) for i in range(0, n - 1, 2)]),
    "phase15_c128": ("f64", lambda n: [("cz", [i, i + 1]) for i in range(0, n - 1, 2)]),
    "tile_h_all": ("f32", lambda n: [("h", [q]) for q in range(13)]),
    "tile_h_all_c128": ("f64", lambda n: [("h", [q]) for q in range(12)]),
    "1q_low_c128": ("f64", lambda n: [("h", [1])]),
    "dense3_c128_high": ("f64", lambda n: [("u3", [n - 16, n - 15, n - 14])]),
    "dense4_c128": ("f64", lambda n: [("u4", [0, 1, 2, 3])]),
    "dense5_c128": ("f64", lambda n: [("u5", [2, 3, 9, 10, 20])]),
    "dense4_c128": ("f64", lambda n: [("u4", [0, 1, 2, 3])]),
    # tensor-core chain passes: one pass of 1 / 2 / 3 Haar 6-qubit matrices on the qubits 0..11; the
    # last matrix leaves qubits 0 and 1 as columns, as the planner arranges in circuits (16-byte
    # staging writes in the epilogue)
    "chain1": ("f32", lambda n: [("u6", list(range(6, 12)))]),
    "chain2": ("f32", lambda n: [("u6", list(range(6, 12))), ("u6", list(range(2, 8)))]),
    "chain3": ("f32", lambda n: [("u6", list(range(6, 12))), ("u6", list(range(6))), ("u6", list(range(3, 9)))]),
}


def run_kernel_case(args):
    """One sweep of one kernel, repeated: per-launch device time and achieved bandwidth."""
    import torch
    from rustatevec_b200 import (B200Backend, Plan, PLAN_AS_GIVEN, PLAN_LEARNED, ENGINE_CUDA_CORE,
                                 ENGINE_TENSOR_CORE)
    from rustatevec_b200 import _lib as L
    from rustatevec_b200 import gate as G
    from rustatevec_b200.circuit import Circuit
    prec, build = KERNEL_CASES[args.kernel_case]
    n = args.qubits
    c = Circuit(n)
    rng = np.random.default_rng(7)
    for name, qs in build(n):
        if name.startswith("u"):
            k = int(name[1:])
            z = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
            q, r = np.linalg.qr(z)
            c.push(G.DenseGate(k, q), qs)
        else:
            c.push(G.LIBRARY[name](), qs)
    engine = ENGINE_TENSOR_CORE if args.kernel_case.startswith("tc") else ENGINE_CUDA_CORE
    planner = PLAN_LEARNED if args.kernel_case.startswith("phase") else PLAN_AS_GIVEN
    if args.kernel_case.startswith("tile"):
        planner = L.PLAN_TILE
    be = B200Backend(0, precision=prec)
    st = be.alloc(n)
    if args.kernel_case.startswith("reduce"):
        be.init_gaussian(st, 7)
        stream = torch.cuda.ExternalStream(be.stream())
        mask = (1 << n) - 1
        for _ in range(2):
            be.expectation_z(st, mask)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.reps):
            be.expectation_z(st, mask)
        e1.record(stream)
        e1.synchronize()
        t = e0.elapsed_time(e1) * 1e-3 / args.reps
        nbytes = float(1 << n) * (16 if prec == "f64" else 8)  # one read of the state
        peak, kind = peaks()
        print(json.dumps({"kernel_case": args.kernel_case, "qubits": n, "precision": prec, "input": "gaussian",
                          "sweeps": ["reduce"], "us_per_call": round(t * 1e6, 2), "algorithmic_bytes": nbytes,
                          "GB/s": round(nbytes / t / 1e9, 1), "frac_of_peak": round(nbytes / t / 1e9 / peak, 4),
                          "peak": f"{peak} ({kind})",
                          "note": "per call: the reduction kernels plus the 16-byte result copy and a synchronize"}))
        st.free()
        be.close()
        return
    # a dense random state by default: a basis state leaves almost every streamed amplitude zero,
    # which draws less power and times optimistically
    if args.input == "basis":
        be.init_basis(st, 0)
    else:
        be.init_gaussian(st, 7)
    opts = L.make_opts(planner, 2, engine, use_graph=False)
    if args.kernel_case.startswith("chain"):
        opts = L.make_opts(L.PLAN_CHAIN, 6, L.ENGINE_AUTO, use_graph=False, chain_max_matrices=3)
    p = Plan(be, c, opts)
    info = p.sweeps()
    stream = torch.cuda.ExternalStream(be.stream())
    for _ in range(2):
        p.run(st)
    be.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.reps):
        p.run(st)
    e1.record(stream)
    e1.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / args.reps
    nbytes = sum(s["algorithmic_bytes"] for s in info)
    peak, kind = peaks()
    print(json.dumps({"kernel_case": args.kernel_case, "qubits": n, "precision": prec, "input": args.input,
                      "sweeps": [s["kind"] for s in info], "us_per_launch": round(t * 1e6, 2),
                      "algorithmic_bytes": nbytes, "GB/s": round(nbytes / t / 1e9, 1),
                      "frac_of_peak": round(nbytes / t / 1e9 / peak, 4), "peak": f"{peak} ({kind})"}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel-case", choices=sorted(KERNEL_CASES))
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--input", default="gaussian", choices=["gaussian", "basis"],
                    help="kernel cases: initial state (dense random, or |0..0>)")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--quick", action="store_true", help="headline plan only")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--ref-budget", type=float, default=10.0)
    ap.add_argument("--no-cpu-scaling", action="store_true", help="skip the full-circuit CPU runs at 24-28 qubits")
    ap.add_argument("--config", default="brickwork30", choices=["brickwork30", "ghz24", "qft32", "qaoa33", "batched"],
                    help="workload (the default is the headline bench line)")
    ap.add_argument("--circuits", type=int, default=4096, help="batched config: number of circuits")
    ap.add_argument("--no-autotune", action="store_true", help="batched config: engine's default tile shape")
    args = ap.parse_args()
    if args.kernel_case:
        run_kernel_case(args)
    elif args.impl == "reference" and args.config == "brickwork30":
        run_reference(args)
    elif args.config == "ghz24":
        run_config_ghz24(args)
    elif args.config == "qft32":
        run_config_qft32(args)
    elif args.config == "qaoa33":
        run_config_qaoa33(args)
    elif args.config == "batched":
        run_config_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
