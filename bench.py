#!/usr/bin/env python
"""Benchmark of the FP64 statevector hot path (driver contract: one JSON line).

Workload (default ``qft30``): the 30-qubit complex128 quantum Fourier
transform (h on qubit j, then cp(pi/2^(k-j)) controlled by every k > j, then
the swap network) preceded by x on a seeded random half of the qubits -- a
16 GiB state, far larger than L2, so every step streams HBM.  One step is one
full ``simulate`` of that circuit: |0...0> initialisation plus every gate.

Metric: effective gate-sweep GB/s = sum over the circuit's gates of the bytes
a per-gate engine must move (2 * 16 B * 2^n * f, f = fraction of amplitudes
the gate changes: 1 for 1q gates, 1/2 for swap/cx, 1/4 for cp) divided by the
step time.  The same definition is used for the CPU reference arm, so the
ratio of the two lines is the speed-up.  ``roofline`` reports the dominant
kernel's own achieved HBM bandwidth (its bytes per launch / its measured
launch time) against the measured copy peak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload qftN|brickwork20]
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import _circuits  # noqa: E402  (workload builders shared with the tests)

PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def peak_hbm():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---- workloads ---------------------------------------------------------------------------

def workload(name: str):
    if name.startswith("qft") and name[3:].isdigit():
        n = int(name[3:])
        if not 10 <= n <= 33:
            raise SystemExit("qftN needs 10 <= N <= 33")
        return _circuits.qft_with_x(n, 1234), {"workload": f"qft{n}_fp64", "num_qubits": n,
                                                "state_bytes": 16 * 2**n,
                                                "circuit": "x(seeded half) + QFT + swap network"}
    if name == "brickwork20":
        return _circuits.brickwork_u3_cx(20, 20, 1234), {"workload": "brickwork20_fp64",
                                                          "num_qubits": 20,
                                                          "state_bytes": 16 * 2**20,
                                                          "circuit": "20 layers u3 + cx brickwork"}
    raise SystemExit(f"unknown workload {name}")


def gate_fraction(kind: str) -> float:
    """Fraction of amplitudes a gate changes (algorithmic bytes per gate)."""
    if kind in ("cp", "cu1", "crz", "cz", "g_cz"):
        return 0.25
    if kind in ("cx", "swap", "cy", "ch", "csx", "crx", "cry", "cu3", "cu", "g_cx"):
        return 0.5
    if kind in ("ccx", "cswap", "rccx"):
        return 0.25
    if kind in ("c3x", "c3sqrtx", "rc3x"):
        return 0.125
    if kind == "c4x":
        return 0.0625
    if kind in ("id", "u0", "barrier", "classical", "g_noop", "g_opaque", "measure", "reset"):
        return 0.0
    return 1.0


def effective_bytes(prog) -> float:
    from dqsim_bosonic_b200._native import KIND_NAMES

    n = prog.num_qubits
    tot = 0.0
    for k in prog.insts["kind"].tolist():
        tot += 2 * 16 * (2 ** n) * gate_fraction(KIND_NAMES[k])
    return tot


# ---- clocks -----------------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        # raw samples go to $DQSIM_CLOCKS_DIR (default: the system temp directory);
        # the JSON line carries their summary
        import tempfile

        base = Path(os.environ.get("DQSIM_CLOCKS_DIR", tempfile.gettempdir()))
        self.path = base / f"dqsim_clocks_dev{device}_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": sorted(reasons)}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---- distributed plumbing ------------------------------------------------------------------------

class Dist:
    def __init__(self, gpus: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", self.local))
            self.pg = dist

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()

    def max(self, v: float) -> float:
        if self.pg is None:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{self.local}")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()


# ---- CPU reference arm / cpu_baseline -------------------------------------------------------------

def _one_inst_program(prog, i):
    sub = prog.insts[i:i + 1].copy()
    sub["cond_count"] = 0
    return type(prog)(sub, prog.conds[:0], prog.num_qubits, 0, max(prog.cbit_space, 1), {})


def _measure_program(prog, qubit):
    from dqsim_bosonic_b200 import _native as nat

    sub = np.zeros(1, dtype=nat.INST_DTYPE)
    sub["kind"] = nat.KIND["measure"]
    sub["nq"] = 1
    sub["q"] = -1
    sub["q"][0, 0] = qubit
    sub["cbit"] = 0
    return type(prog)(sub, prog.conds[:0], prog.num_qubits, 1, 1, {})


class CpuClassTimer:
    """Times the restated reference engine (oracle, OpenMP) per gate class of
    the workload on the full host state, and extrapolates to the whole
    program: t_program = sum over classes of count_class x mean time of a
    gate of that class (engine.rs:43-87 one-qubit loop, :127-156 n-qubit
    filter, :197-235 measure).  One measure is timed beside the gates and
    reported, not extrapolated (the program has none)."""

    def __init__(self, prog, threads: int):
        import _oracle
        from dqsim_bosonic_b200._native import KIND_NAMES

        self.orc = _oracle
        self.prog = prog
        self.threads = threads
        n = prog.num_qubits
        self.state = np.empty(1 << n, dtype=np.complex128)
        self.state[:] = 1.0 / math.sqrt(self.state.size)  # touch every page before timing
        kinds = [KIND_NAMES[k] for k in prog.insts["kind"].tolist()]
        self.members = {}
        for i, k in enumerate(kinds):
            if gate_fraction(k) > 0.0:
                self.members.setdefault(k, []).append(i)
        self.count = {k: len(v) for k, v in self.members.items()}
        self.times = {k: [] for k in self.members}
        self.measure_times = []
        self.cursor = {k: 0 for k in self.members}

    def _time(self, p) -> float:
        t0 = time.perf_counter()
        self.orc.run_inplace(p, 0, self.state)
        return time.perf_counter() - t0

    def sample(self, per_class: int, record: bool = True) -> float:
        """Time `per_class` gates of every class (cycling through the
        program's own instances) and one measure; returns the wall seconds."""
        self.orc.set_threads(self.threads)
        wall = 0.0
        for k in sorted(self.members):
            idx = self.members[k]
            for _ in range(per_class):
                i = idx[self.cursor[k] % len(idx)]
                self.cursor[k] += 1
                dt = self._time(_one_inst_program(self.prog, i))
                wall += dt
                if record:
                    self.times[k].append(dt)
        dt = self._time(_measure_program(self.prog, 0))
        wall += dt
        if record:
            self.measure_times.append(dt)
        # the measurement halved the support: restore the uniform state
        self.state[:] = 1.0 / math.sqrt(self.state.size)
        self.orc.set_threads(1)
        return wall

    def program_seconds(self) -> float:
        return sum(self.count[k] * float(np.mean(v)) for k, v in self.times.items())

    def gates_timed(self) -> int:
        return sum(len(v) for v in self.times.values())

    def report(self) -> dict:
        return {
            "per_class_ms": {k: round(1e3 * float(np.mean(v)), 3) for k, v in sorted(self.times.items())},
            "class_counts": dict(sorted(self.count.items())),
            "gates_timed": self.gates_timed(),
            "measure_ms": round(1e3 * float(np.mean(self.measure_times)), 3) if self.measure_times else None,
            "extrapolated_program_s": self.program_seconds(),
        }

    def sample_text(self) -> str:
        n = self.prog.num_qubits
        classes = ", ".join(f"{k} x{len(v)}" for k, v in sorted(self.times.items()))
        return (f"{self.gates_timed()} gates ({classes}) + {len(self.measure_times)} measure on the "
                f"full {n}-qubit state, extrapolated per class to the {int(self.prog.ninst)}-instruction "
                f"program; restated reference engine (oracle/liboracle.so)")


def run_reference_arm(args, wl_prog, cfg):
    dist_rank = int(os.environ.get("RANK", "0"))
    if dist_rank != 0:
        return
    threads = os.cpu_count() or 1
    timer = CpuClassTimer(wl_prog, threads)
    # at least 20 timed gates over the run, spread over its steps
    per_class = max(1, math.ceil(20 / (max(len(timer.members), 1) * max(args.steps, 1))))
    for _ in range(args.warmup):
        timer.sample(1, record=False)
    walls = []
    for _ in range(args.steps):
        walls.append(timer.sample(per_class))
    t_prog = timer.program_seconds()
    eff = effective_bytes(wl_prog)
    value = eff / t_prog / 1e9
    line = {
        "impl": "reference",
        "metric": "effective gate-sweep GB/s (FP64 statevector)",
        "value": value,
        "unit": "GB/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": float(np.mean(walls) * 1000.0),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded circuit)",
        "config": cfg,
        "step_note": "one step = one bounded sample: every gate class of the workload timed on the full "
                     "state; value = the workload's effective bytes / the per-class extrapolation of "
                     "the whole program",
        "cpu_baseline": dict({"value": value, "unit": "GB/s", "cores": threads, "kind": "port",
                              "sample": timer.sample_text()}, **timer.report()),
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- our arm ------------------------------------------------------------------------------------------

def profile_case(spec: str) -> None:
    """One small case of one kernel (no JSON line): the command a profiler wraps."""
    kind, *rest = spec.split(":")
    if kind == "ragged":
        from dqsim_bosonic_b200.batch import run_batch
        from dqsim_bosonic_b200.circuit import decode_program

        n, count = int(rest[0]), int(rest[1])
        circs = _circuits.ragged_batch(1024, 99)
        progs = [decode_program(c.model_dump_json()) for c in circs]
        idx = [k for k, p in enumerate(progs) if p.num_qubits == n][:count]
        for _ in range(2):
            _, _, st = run_batch([progs[k] for k in idx], [99 + k for k in idx], 0)
        print(f"ragged n={n} items={len(idx)} kernel_ms={st.kernel_ms:.3f} launches={st.launches}")
    elif kind == "adjoint":
        from dqsim_bosonic_b200.adjoint import adjoint_gradient

        n = int(rest[0])
        c, theta, H = _circuits.hea_param_circuit(n, 16, seed=1)
        for _ in range(2):
            tm = {}
            adjoint_gradient(c, theta, H, device=0, timing=tm)
        print(f"adjoint n={n} " + " ".join(f"{k}={v}" for k, v in tm.items()))
    elif kind == "merge":
        n = int(rest[0])
        r = pblock_merge_section(0, n)
        print(f"merge n={n} ms={r['ms']:.4f} frac={r['roofline']['frac']:.4f}")
    else:
        raise SystemExit(f"unknown profile case {spec!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="qft30")
    ap.add_argument("--exec", default=None, choices=[None, "fused", "per_gate"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the trajectory-batch and adjoint-gradient sections")
    ap.add_argument("--adam-steps", type=int, default=2,
                    help="timed Adam steps of the 512-set batched adjoint (0 = skip)")
    ap.add_argument("--merge-qubits", type=int, default=30,
                    help="qubits of the merged block in the p-block merge section (even split)")
    ap.add_argument("--no-adjoint31", action="store_true",
                    help="skip the 31-qubit adjoint pass with its finite-difference check")
    ap.add_argument("--profile-case", default=None,
                    help="run one small case of one kernel for a profiler and exit: "
                         "ragged:<n>:<items> (run_batch over the first <items> items of <n> "
                         "qubits of the 1024-circuit ragged set, twice), adjoint:<n> "
                         "(two adjoint gradients of the 16-layer ansatz on <n> qubits) or "
                         "merge:<n> (the merge section's 3 warm-up and 5 timed block merges "
                         "into an <n>-qubit block)")
    args = ap.parse_args()
    if args.profile_case:
        profile_case(args.profile_case)
        return

    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

    circ, cfg = workload(args.workload)
    prog = encode(decode_circuit_json(circ.model_dump_json()))
    cfg = dict(cfg)
    cfg.update({"gates": int(prog.ninst), "parallelism": f"replicas x{args.gpus}",
                "l2": "state larger than L2 (126 MB)" if cfg["state_bytes"] > 126e6 else
                      "state L2-resident; L2 flushed between steps"})

    if args.impl == "reference":
        run_reference_arm(args, prog, cfg)
        return

    import ctypes

    import torch

    from dqsim_bosonic_b200 import StatevectorSimulator
    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.statevector import run_program

    d = Dist(args.gpus)
    dev = d.local
    torch.cuda.set_device(dev)
    exec_mode = nat.EXEC_PER_GATE if args.exec == "per_gate" else nat.EXEC_FUSED
    if args.exec is None:
        exec_mode = nat.EXEC_FUSED if os.environ.get("DQSIM_EXEC", "fused") == "fused" else nat.EXEC_PER_GATE
    eff_bytes = effective_bytes(prog)
    flush = None
    if cfg["state_bytes"] <= 126e6:
        flush = torch.empty(256 * 2**20, dtype=torch.uint8, device=f"cuda:{dev}")

    # ---- value: device-timed steps, program resident, state in HBM ----
    st = nat.State(prog.num_qubits, dev)
    ptr, sptr = st.device_ptr()
    stream = torch.cuda.ExternalStream(sptr, device=f"cuda:{dev}")
    launches = 0

    def step():
        nonlocal launches
        st.reset()
        _, prof = run_program(st, prog, 7, nat.SEM_SIMULATE, exec_mode)
        launches += int(prof.kernel_launches)
        return prof

    for _ in range(max(args.warmup, 3)):
        step()
    if flush is not None:
        flush.zero_()
    torch.cuda.synchronize(dev)
    d.barrier()
    torch.cuda.synchronize(dev)
    launches = 0
    ev = []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            if flush is not None:
                with torch.cuda.stream(stream):
                    flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prof = step()
            e1.record(stream)
            ev.append((e0, e1))
        torch.cuda.synchronize(dev)
    d.barrier()
    torch.cuda.synchronize(dev)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = d.max(float(np.sum(step_ms)))
    ms_per_step = total_ms / args.steps
    value = eff_bytes * args.steps * d.world / (total_ms * 1e-3) / 1e9
    sweeps = int(prof.sweeps)

    # ---- dominant kernel roofline: time its launches with events on its stream ----
    roof = dominant_kernel_roofline(st, prog, exec_mode, stream, dev)
    st.release()

    # ---- e2e: public API with host circuit in, probabilities out ----
    sim = StatevectorSimulator(seed=7, device=dev,
                               exec="per_gate" if exec_mode == nat.EXEC_PER_GATE else "fused")
    n = prog.num_qubits
    top = list(range(n - 1, max(-1, n - 11), -1))
    # the interpreter's cyclic garbage collector stays off inside the timed
    # host steps (as timeit does); it runs between them.  The untimed warm-up
    # steps run exactly like the timed ones (a freshly started box is noisy
    # for a while, and the first step after a collection was slow).
    gc.collect()
    for _ in range(max(5, args.warmup)):
        torch.cuda.synchronize(dev)
        gc.disable()
        res = sim.simulate(circ)
        res.probabilities(top)
        torch.cuda.synchronize(dev)
        gc.enable()
        del res
        gc.collect()
    d.barrier()
    e2e_t, phases = [], []
    for _ in range(args.steps):
        torch.cuda.synchronize(dev)
        gc.disable()
        t0 = time.perf_counter()
        res = sim.simulate(circ)
        p = res.probabilities(top)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t0
        e2e_t.append(dt)
        ph = dict(res.timings)
        ph["other_ms"] = dt * 1e3 - (ph["parse_ms"] + ph["state_ms"] + ph["run_ms"] + ph["query_ms"])
        phases.append({k: round(v, 3) for k, v in ph.items()})
        gc.enable()
        del res, p
        gc.collect()
    e2e_total = d.max(float(np.sum(e2e_t)))
    e2e_value = eff_bytes * args.steps * d.world / e2e_total / 1e9

    line = {
        "metric": "effective gate-sweep GB/s (FP64 statevector)",
        "value": value,
        "unit": "GB/s",
        "n_gpus": d.world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_per_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded circuit)",
        "config": cfg,
        "exec": "fused" if exec_mode == nat.EXEC_FUSED else "per_gate",
        "sweeps_per_step": sweeps,
        "e2e": {"value": e2e_value, "unit": "GB/s",
                "h2d_bytes_per_step": int(prog.insts.nbytes + prog.conds.nbytes),
                "d2h_bytes_per_step": int(8 * (1 << len(top))),
                "ms_per_step": e2e_total / args.steps * 1000.0,
                "median_step_ms": float(np.median(e2e_t)) * 1e3,
                "step_ms": [round(1e3 * x, 3) for x in e2e_t],
                "phases_ms": phases,
                "phases_note": "per step: parse = JSON decode + encode, state = handle + buffer from "
                               "the cache, run = dq_run (returns when the state is final), engine = "
                               "the engine's clock inside dq_run, query = probabilities(), other = "
                               "the rest of the step",
                "path": "StatevectorSimulator.simulate(circuit) + probabilities(top 10 qubits)"},
        "roofline": roof,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if not args.no_extras:
        line["trajectories"] = trajectory_section(dev, cpu=d.rank == 0 and d.world == 1
                                                  and not args.no_cpu_baseline, d=d)
        line["adjoint"] = adjoint_section(dev)
        line["pblock_merge"] = pblock_merge_section(dev, args.merge_qubits)
        line["mps"] = mps_section(dev, cpu=d.rank == 0 and d.world == 1 and not args.no_cpu_baseline)
        if args.adam_steps > 0:
            line["adjoint_batch"] = adjoint_batch_section(dev, args.adam_steps)
    if not args.no_extras:
        line["distributed30"] = distributed30_section(dev, args.steps)
        line["ragged"] = ragged_section(dev, cpu=d.rank == 0 and d.world == 1
                                        and not args.no_cpu_baseline)
    if not args.no_extras and not args.no_adjoint31:
        line["adjoint31"] = adjoint31_section(dev)
    if "_cpu_job" in line.get("trajectories", {}):
        trajectory_cpu_baseline(line["trajectories"])
    if d.rank == 0 and d.world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        timer = CpuClassTimer(prog, threads)
        timer.sample(1, record=False)
        per_class = max(1, math.ceil(20 / max(len(timer.members), 1)))
        timer.sample(per_class)
        line["cpu_baseline"] = dict({"value": eff_bytes / timer.program_seconds() / 1e9, "unit": "GB/s",
                                     "cores": threads, "kind": "port",
                                     "sample": timer.sample_text()}, **timer.report())
    if d.rank == 0:
        print(json.dumps(line), flush=True)
    d.close()


def trajectory_section(dev: int, cpu: bool, d=None) -> dict:
    """4096 shots of the 16-qubit trajectory workload (12 layers of u3 + cx
    brickwork, measure / conditional x / reset after every third layer) in one
    persistent launch replayed from a CUDA graph, against per-shot launches of
    the plain per-gate kernels on the same GPU and the oracle on the host.
    With N ranks every rank runs 4096 shots of its own slice of the global
    shot range (weak scaling: seeds base + global shot index) and the counts
    are merged with one all-reduce of the outcome histogram."""
    from dqsim_bosonic_b200 import StatevectorSimulator
    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.batch import TrajectoryPlan, TrajectoryTuner
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from dqsim_bosonic_b200.statevector import run_program

    from dqsim_bosonic_b200.circuit import format_cbits
    from dqsim_bosonic_b200.dist import merge_counts, shard_range

    world = d.world if d is not None else 1
    rank = d.rank if d is not None else 0
    shots, base_seed = 4096, 7
    circ = _circuits.trajectory_circuit(16, 12, seed=7)
    prog = encode(decode_circuit_json(circ.model_dump_json()))
    tuner = TrajectoryTuner(trial_shots=512)
    opts = tuner.choose(prog, dev)
    plan = TrajectoryPlan(prog, shots, dev, opts=opts)
    lo, _ = shard_range(shots * world, rank, world)
    for _ in range(2):
        plan.run(base_seed + lo)
    ms = []
    for _ in range(5):
        bits, st = plan.run(base_seed + lo)
        ms.append(st.kernel_ms)
    kernel_ms = float(np.median(ms))
    if d is not None:
        kernel_ms = d.max(kernel_ms)
    local = {}
    for row in bits:
        k = format_cbits(row, prog.num_cbits)
        local[k] = local.get(k, 0) + 1
    merged = merge_counts(local, prog.num_cbits)
    # per-shot launches of the exact per-gate kernels (HBM-resident state)
    state = nat.State(16, dev)
    k = 16
    run_program(state, prog, base_seed, nat.SEM_SHOTS, nat.EXEC_PER_GATE)
    t0 = time.perf_counter()
    for i in range(k):
        state.reset()
        run_program(state, prog, base_seed + i, nat.SEM_SHOTS, nat.EXEC_PER_GATE)
    per_shot_ms = (time.perf_counter() - t0) * 1e3 / k
    state.release()
    # e2e through the public API (JSON circuit in, counts out)
    sim = StatevectorSimulator(seed=base_seed, device=dev)
    sim.simulate_shots(circ, shots)
    t0 = time.perf_counter()
    sim.simulate_shots(circ, shots)
    e2e_ms = (time.perf_counter() - t0) * 1e3
    out = {
        "workload": "4096 shots x 16 qubits per GPU, 12 layers u3+cx brickwork, "
                    "measure/cond-x/reset every 3rd layer (base_seed 7)",
        "kernel_ms": kernel_ms,
        "shots_per_s": shots * world / (kernel_ms * 1e-3),
        "ranks": world,
        "merged_counts": merged,
        "e2e_ms": e2e_ms,
        "e2e_path": "StatevectorSimulator.simulate_shots(circuit, 4096)",
        "per_shot_launches_ms": per_shot_ms * shots,
        "per_shot_launches_note": f"plain per-gate kernels, one shot at a time; {k} shots timed, x{shots // k}",
        "speedup_vs_per_shot_launches": per_shot_ms * shots / kernel_ms,
        "geometry": {"threads": int(opts.threads or 256), "local_bits": int(st.local_bits),
                     "cluster_span": int(st.cluster_span), "clusters": int(st.clusters)},
        "boundary_draws": int(st.boundary_draws),
        "hbm_bytes": 0,
    }
    if cpu:
        # the oracle sample runs after every GPU section (its OpenMP threads
        # must not share the host with timed GPU work): keep what it needs
        out["_cpu_job"] = (prog, base_seed, bits, int(st.boundary_draws))
    plan.release()
    return out


def trajectory_cpu_baseline(traj: dict) -> None:
    """The oracle's shots/s on 256 shots of the trajectory workload and their
    parity with the GPU's first 256 shots (filled into the trajectory section)."""
    import _oracle as orc

    prog, base_seed, bits, boundary = traj.pop("_cpu_job")
    threads = os.cpu_count() or 1
    orc.set_threads(threads)
    m = 256
    t0 = time.perf_counter()
    want, rc, _ = orc.run_shots(prog, base_seed, m)
    cpu_s = time.perf_counter() - t0
    orc.set_threads(1)
    bad = int(np.sum(np.any(bits[:m] != want, axis=1)))
    traj["cpu_baseline"] = {"shots_per_s": m / cpu_s, "cores": threads, "kind": "port",
                            "sample": f"{m} shots on the oracle (sequential per shot)"}
    traj["parity"] = {"shots_checked": m, "mismatches": bad, "allowed_boundary_draws": boundary}


def adjoint_section(dev: int) -> dict:
    """24-qubit hardware-efficient ansatz, 16 layers (1152 parameters),
    H = sum a_i Z_i Z_{i+1} + sum b_i X_i: adjoint gradient vs GPU parameter
    shift (2 forward runs per parameter with the plain per-gate kernels)."""
    from dqsim_bosonic_b200.adjoint import adjoint_gradient, expectation, parameter_shift_gradient

    c, theta, H = _circuits.hea_param_circuit(24, 16, seed=1)
    adjoint_gradient(c, theta, H, device=dev)
    reps, times, tms = 5, [], []
    for _ in range(reps):
        tm = {}
        t0 = time.perf_counter()
        e, g = adjoint_gradient(c, theta, H, device=dev, timing=tm)
        times.append(time.perf_counter() - t0)
        tms.append(tm)
    t_adj = float(np.median(times))
    tm = tms[int(np.argsort(times)[len(times) // 2])]
    # forward runs of the parameter-shift baseline: the fastest of three (a
    # host stall during one run must not inflate the baseline)
    fwd = {}
    for ex in ("per_gate", "fused"):
        expectation(c, theta, H, device=dev, exec=ex)
        ts = []
        for _ in range(3):
            t0 = time.perf_counter()
            expectation(c, theta, H, device=dev, exec=ex)
            ts.append(time.perf_counter() - t0)
        fwd[ex] = min(ts)
    P = theta.size
    sub = list(range(0, P, P // 8))[:8]
    ps = parameter_shift_gradient(c, theta, H, device=dev, exec="per_gate", occurrences=sub)
    err = float(np.max(np.abs(g[sub] - ps[sub])))
    n = c.num_qubits
    # per-gate algorithmic bytes (psi and lambda read + written per gate) and
    # the bytes the fused sweeps actually stream (once per sweep)
    gate_bytes = len(c.ops) * 64.0 * 2 ** n
    sweeps = int(tm["backward_sweeps"])
    back_bytes = sweeps * 64.0 * 2 ** n
    peak, src = peak_hbm()
    achieved = back_bytes / (tm["backward_ms"] * 1e-3) / 1e9
    ps_s = 2 * P * fwd["per_gate"]
    return {
        "workload": "hea24: 16 layers (ry, rz on all qubits, rzz ring), 1152 params; "
                    "H = sum a_i Z_i Z_i+1 + sum b_i X_i",
        "ms_per_gradient": t_adj * 1e3,
        "grads_per_s": 1.0 / t_adj,
        "phases_ms": tm,
        "expval": e,
        "param_shift_ms_per_gradient": ps_s * 1e3,
        "param_shift_note": "2 x 1152 forward runs (plain per-gate kernels) + <H>; fastest of 3 forward runs, x2P",
        "speedup_vs_param_shift": ps_s / t_adj,
        "param_shift_fused_forward_ms_per_gradient": 2 * P * fwd["fused"] * 1e3,
        "speedup_vs_fused_param_shift": 2 * P * fwd["fused"] / t_adj,
        "max_abs_diff_vs_param_shift": err,
        "params_checked": len(sub),
        "backward_roofline": {"kernel": "k_adj_sweep (fused backward sweep over psi and lambda)",
                              "bound": "hbm", "sweeps": sweeps,
                              "bytes_per_launch": 64.0 * 2 ** n, "achieved": achieved,
                              "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                              "peak_source": src,
                              "effective_gate_gbs": gate_bytes / (tm["backward_ms"] * 1e-3) / 1e9,
                              "effective_note": "per-gate algorithmic bytes (64 B x 2^n per gate) "
                                                "over the backward time; above the HBM peak "
                                                "because fused gates share one pass"},
    }


def adjoint_batch_section(dev: int, adam_steps: int) -> dict:
    """512 parameter sets of the 20-qubit, 8-layer ansatz (480 parameters
    each) through the torch autograd function, driving Adam (lr 0.01) on the
    sum of the energies.  Every set's gradient comes from one batched adjoint
    call per step (dq_adjoint_batch: each forward sweep, lambda = H psi and
    each backward sweep is one launch over all 512 sets).  Times `adam_steps`
    steps after one warm-up step."""
    import torch

    from dqsim_bosonic_b200.adjoint import adjoint_gradient_batch, expval

    c, theta, H = _circuits.hea_param_circuit(20, 8, seed=1)
    B = 512
    rng = np.random.default_rng(11)
    t = torch.tensor(rng.uniform(-math.pi, math.pi, size=(B, c.num_params)), requires_grad=True)
    opt = torch.optim.Adam([t], lr=0.01)

    def step():
        opt.zero_grad()
        e = expval(t, c, H, device=dev)
        e.sum().backward()
        opt.step()
        return e.detach()

    e0 = step()
    t0 = time.perf_counter()
    for _ in range(adam_steps):
        e = step()
    dt = (time.perf_counter() - t0) / max(adam_steps, 1)
    st = {}
    adjoint_gradient_batch(c, t.detach().numpy(), H, device=dev, stats=st)
    return {
        "workload": "512 parameter sets x hea20 (8 layers, 480 params), Adam lr 0.01 on sum <H>",
        "s_per_adam_step": dt,
        "gradients_per_s": B / dt,
        "adam_steps_timed": adam_steps,
        "projected_s_for_50_steps": 50 * dt,
        "mean_energy_first": float(e0.mean()),
        "mean_energy_last": float(e.mean()),
        "launches_per_gradient_batch": int(st["launches"]),
        "forward_sweeps": int(st["forward_sweeps"]),
        "backward_sweeps": int(st["backward_sweeps"]),
        "phases_ms": {"plan": st["plan_ms"], "forward": st["forward_ms"],
                      "observable": st["observable_ms"], "backward": st["backward_ms"]},
        "batched": bool(st["batched"]),
        "set_groups": int(st["groups"]),
    }


def pblock_merge_section(dev: int, n: int = 30) -> dict:
    """The p-block merge of two blocks on the even and the odd qubits into an
    n-qubit block (n = 30: two 15-qubit blocks): dq_block_merge timed with
    CUDA events on the merged state's stream; algorithmic bytes = the merged
    state written plus both blocks read."""
    import torch

    from dqsim_bosonic_b200 import _native as nat

    qa = np.arange(0, n, 2, dtype=np.uint32)
    qb = np.arange(1, n, 2, dtype=np.uint32)
    na, nb = int(qa.size), int(qb.size)
    sa, sb, out = nat.State(na, dev), nat.State(nb, dev), nat.State(n, dev)
    rng = np.random.default_rng(3)
    for s_, k in ((sa, na), (sb, nb)):
        v = rng.normal(size=1 << k) + 1j * rng.normal(size=1 << k)
        s_.upload(v / np.linalg.norm(v))
    _, sptr = out.device_ptr()
    stream = torch.cuda.ExternalStream(sptr, device=f"cuda:{dev}")
    L = nat.lib()

    def merge():
        nat.check(L.dq_block_merge(sa.handle, nat.ptr(qa), na, sb.handle, nat.ptr(qb), nb, out.handle),
                  "dq_block_merge")

    for _ in range(3):
        merge()
    ms = []
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        merge()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    for s_ in (sa, sb, out):
        s_.release()
    t = float(np.median(ms))
    nbytes = 16.0 * (2 ** n + 2 ** na + 2 ** nb)
    peak, src = peak_hbm()
    achieved = nbytes / (t * 1e-3) / 1e9
    return {"workload": f"merge_blocks: {na} + {nb} interleaved qubits -> {n}-qubit block",
            "ms": t, "bytes": nbytes,
            "roofline": {"kernel": "k_block_merge", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": src}}


def mps_section(dev: int, cpu: bool) -> dict:
    """The MPS backend (MpsSimulator): (a) the 16-qubit trajectory workload
    (12 layers of u3 + cx brickwork, measure / conditional x / reset every
    third layer) as 4096 MPS shots with max_bond_dimension 16, one batch of
    independent MPS per launch; (b) one `simulate` of the 20-qubit u3 + cx
    brickwork (20 layers) with max_bond_dimension 64 (single MPS: the SVD
    steps run one after another).  CPU baseline: the numpy MPS oracle
    (oracle/mps.py, LAPACK SVD) on a sample, with its cbits / statevector
    compared to the device's."""
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from dqsim_bosonic_b200.mps import MpsHandle, run_mps_shots

    out = {}
    prog = encode(decode_circuit_json(_circuits.trajectory_circuit(16, 12, seed=7).model_dump_json()))
    shots, chi = 4096, 16
    run_mps_shots(prog, 7, 256, dev, chi, 1e-12)
    walls, sts = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        bits, st = run_mps_shots(prog, 7, shots, dev, chi, 1e-12)
        walls.append(time.perf_counter() - t0)
        sts.append(st)
    i = int(np.argsort(walls)[1])
    wall, st = walls[i], sts[i]
    traj = {"workload": "MPS shots: 16-qubit trajectory circuit, 12 layers, measure/cond/reset, "
                        f"{shots} shots, max_bond_dimension {chi}",
            "shots_per_s": shots / wall, "wall_ms": wall * 1e3, "kernel_ms": st.kernel_ms,
            "svd_steps": int(st.svd_calls), "svd_steps_per_s": st.svd_calls / (st.kernel_ms * 1e-3),
            "replicas_per_launch": int(st.replicas), "bond_capacity": int(st.capacity)}
    if cpu:
        import _oracle as orc

        m = 16
        t0 = time.perf_counter()
        bad = 0
        for k in range(m):
            _, cb, _, _ = orc.mps_run(prog, 7 + k, max_bond=chi)
            bad += int(cb[:prog.cbit_space].tolist() != bits[k].tolist())
        cpu_s = time.perf_counter() - t0
        traj["cpu_baseline"] = {"shots_per_s": m / cpu_s, "cores": 1, "kind": "port",
                                "sample": f"{m} shots on the numpy MPS oracle (LAPACK SVD)"}
        traj["parity"] = {"shots_checked": m, "cbit_mismatches": bad}
    out["trajectories"] = traj

    n, layers, chi1 = 20, 20, 64
    prog1 = encode(decode_circuit_json(_circuits.brickwork_u3_cx(n, layers, seed=1234).model_dump_json()))
    h = MpsHandle(n, dev, chi1, 1e-12)
    h.run(prog1, 1)
    ts = []
    for _ in range(3):
        t0 = time.perf_counter()
        _, st1 = h.run(prog1, 1)
        ts.append(time.perf_counter() - t0)
    dims = h.bond_dims()
    sv = h.to_state().download() if cpu else None
    h.release()
    single = {"workload": f"MpsSimulator.simulate: {n}-qubit u3+cx brickwork, {layers} layers, "
                          f"max_bond_dimension {chi1}",
              "wall_ms": float(np.median(ts)) * 1e3, "kernel_ms": st1.kernel_ms,
              "svd_steps": int(st1.svd_calls), "us_per_svd_step": st1.kernel_ms * 1e3 / max(st1.svd_calls, 1),
              "max_bond": int(max(dims))}
    if cpu:
        import _oracle as orc

        t0 = time.perf_counter()
        ref, _, rdims, _ = orc.mps_run(prog1, 1, max_bond=chi1)
        cpu_s = time.perf_counter() - t0
        single["cpu_baseline"] = {"wall_ms": cpu_s * 1e3, "cores": 1, "kind": "port",
                                  "sample": "the same simulate on the numpy MPS oracle (LAPACK SVD)"}
        single["parity"] = {"max_abs_amplitude_diff": float(np.max(np.abs(sv - ref))),
                            "bond_dims_equal": rdims == dims}
    out["simulate"] = single
    return out


def ragged_section(dev: int, cpu: bool) -> dict:
    """1024 independent u3 + cx brickwork circuits, n ~ U{10..22} qubits,
    depth ~ U{5..40} layers (seed 99), one trajectory each through
    dq_run_batch: ONE persistent launch (states of <= 16 qubits in cluster
    shared memory, 17..22 qubits HBM-resident fused sweeps).  Against
    per-circuit launches of the fused engine on the same GPU (a seeded sample
    of 64 circuits, scaled to the batch) and, for parity, the final states of
    a sample of items compared with the oracle."""
    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.batch import run_batch
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from dqsim_bosonic_b200.statevector import run_program

    circs = _circuits.ragged_batch(1024, 99)
    progs = [encode(decode_circuit_json(c.model_dump_json())) for c in circs]
    seeds = [99 + k for k in range(len(progs))]
    ns = np.array([p.num_qubits for p in progs])
    run_batch(progs, seeds, dev)  # warm-up (module load, allocations)
    walls, sts = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        _, _, st = run_batch(progs, seeds, dev)
        walls.append(time.perf_counter() - t0)
        sts.append(st)
    i = int(np.argsort(walls)[1])
    wall, st = walls[i], sts[i]
    # per-circuit launches of the fused engine (HBM state per circuit), sample scaled up
    rng = np.random.default_rng(7)
    sample = rng.choice(len(progs), size=64, replace=False)
    states = {}
    for k in sample:
        p = progs[k]
        s = states.get(p.num_qubits)
        if s is None:
            s = states[p.num_qubits] = nat.State(p.num_qubits, dev)
        s.reset()
        run_program(s, p, seeds[k], nat.SEM_SHOTS, nat.EXEC_FUSED)
    per = 0.0
    for k in sample:
        p = progs[k]
        s = states[p.num_qubits]
        t0 = time.perf_counter()
        s.reset()
        run_program(s, p, seeds[k], nat.SEM_SHOTS, nat.EXEC_FUSED)
        per += time.perf_counter() - t0
    for s in states.values():
        s.release()
    per_batch_s = per * len(progs) / len(sample)
    out = {"workload": "1024 u3+cx brickwork circuits, n ~ U{10..22}, depth ~ U{5..40} layers (seed 99)",
           "items": len(progs), "qubit_histogram": {int(q): int((ns == q).sum()) for q in np.unique(ns)},
           "wall_ms": wall * 1e3, "kernel_ms": st.kernel_ms, "items_per_s": len(progs) / wall,
           "launches": int(st.launches), "hbm_items": int(st.hbm_items),
           "engine_items": int(st.engine_items), "cluster_span": int(st.cluster_span),
           "clusters": int(st.clusters),
           "per_circuit_launches_s": per_batch_s,
           "per_circuit_note": "one fused dq_run per circuit (64 sampled circuits, scaled to 1024)",
           "speedup_vs_per_circuit": per_batch_s / wall}
    if cpu:
        import _oracle as orc

        pick = [int(k) for k in np.argsort(ns * 1000 + np.arange(len(ns)))[:6]]
        pick += [int(k) for k in np.flatnonzero((ns >= 17) & (ns <= 18))[:2]]
        _, sv, _ = run_batch(progs, seeds, dev, want_states=pick)
        worst = 0.0
        for k in pick:
            ref, _, rc, _ = orc.run(progs[k], 0)
            worst = max(worst, float(np.max(np.abs(sv[k] - ref))))
        out["parity"] = {"items_checked": len(pick), "qubits": [int(ns[k]) for k in pick],
                         "max_abs_amplitude_diff": worst, "tolerance": 1e-12}
    return out


def distributed30_section(dev: int, steps: int) -> dict:
    """The two-node distributed variant of the 30-qubit workload: node A data
    qubits 0..13 + link 14, node B link 15 + data 16..29, remote_link_psi_minus
    on the links and nonlocal_cz across the nodes, lowered to one 30-qubit
    circuit (generic gate arms of statevector/simulator.rs:571-600).  Device
    time of the fused run (CUDA events on the state's stream) and the public
    API end to end (simulate + probabilities of the top 10 qubits)."""
    import torch

    from dqsim_bosonic_b200 import StatevectorSimulator
    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from dqsim_bosonic_b200.statevector import run_program

    circ = _circuits.distributed_qft_variant(14, 1234)
    prog = encode(decode_circuit_json(circ.model_dump_json()))
    n = prog.num_qubits
    st = nat.State(n, dev)
    _, sptr = st.device_ptr()
    stream = torch.cuda.ExternalStream(sptr, device=f"cuda:{dev}")
    for _ in range(3):
        st.reset()
        run_program(st, prog, 7, nat.SEM_SIMULATE, nat.EXEC_FUSED)
    ms = []
    for _ in range(max(steps, 3)):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st.reset()
        _, prof = run_program(st, prog, 7, nat.SEM_SIMULATE, nat.EXEC_FUSED)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    st.release()
    sim = StatevectorSimulator(seed=7, device=dev, exec="fused")
    top = list(range(n - 1, n - 11, -1))
    for _ in range(2):
        sim.simulate(circ).probabilities(top)
    e2e = []
    for _ in range(max(steps, 3)):
        t0 = time.perf_counter()
        res = sim.simulate(circ)
        res.probabilities(top)
        e2e.append(time.perf_counter() - t0)
        del res
    t = float(np.median(ms))
    eff = effective_bytes(prog)
    return {"workload": "2 x 14 data + 2 link qubits (30), remote_link_psi_minus + nonlocal_cz, "
                        "lowered to one circuit", "gates": int(prog.ninst), "ms": t,
            "effective_gbs": eff / (t * 1e-3) / 1e9, "sweeps": int(prof.sweeps),
            "kernel_launches": int(prof.kernel_launches),
            "e2e_ms": float(np.median(e2e)) * 1e3,
            "parity": "tests/test_gpu_headline.py: fused vs the exact per-gate engine over all 2^30 "
                      "amplitudes, within 1e-12"}


def adjoint31_section(dev: int, fd_params: int = 32) -> dict:
    """One adjoint pass at 31 qubits (4 layers, 372 parameters; psi and lambda
    = 64 GiB in HBM), gradient checked by central differences (h = 1e-6) on a
    seeded subset of parameters."""
    from dqsim_bosonic_b200.adjoint import adjoint_gradient, expectation

    c, theta, H = _circuits.hea_param_circuit(31, 4, seed=1)
    tm = {}
    t0 = time.perf_counter()
    e, g = adjoint_gradient(c, theta, H, device=dev, timing=tm)
    t_adj = time.perf_counter() - t0
    sub = sorted(np.random.default_rng(0).choice(theta.size, size=fd_params, replace=False).tolist())
    h = 1e-6
    fd = []
    for k in sub:
        tp = theta.copy(); tp[k] += h
        tmn = theta.copy(); tmn[k] -= h
        fd.append((expectation(c, tp, H, device=dev) - expectation(c, tmn, H, device=dev)) / (2 * h))
    err = float(np.max(np.abs(np.array(fd) - g[sub])))
    return {"workload": "hea31: 4 layers, 372 params", "s_per_gradient": t_adj, "phases_ms": tm,
            "expval": e, "fd_params": len(sub), "fd_h": h, "max_abs_diff_vs_fd": err}


def dominant_kernel_roofline(st, prog, exec_mode, stream, dev):
    """Time the kernel that dominates the step and report its HBM roofline."""
    import torch

    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

    peak, src = peak_hbm()
    n = prog.num_qubits
    reps = 3
    if exec_mode == nat.EXEC_FUSED:
        name, nbytes, ms = fused_sweep_timing(st, prog, stream, reps)
    else:
        # per-gate path: cp (k_phase) carries most of the time in the QFT
        one = encode(decode_circuit_json(_circuits.JsonCircuit(
            n, [_circuits.g("cp", n - 1, n // 2, 0.3)]).model_dump_json()))
        from dqsim_bosonic_b200.statevector import run_program

        run_program(st, one, 0, nat.SEM_SIMULATE, nat.EXEC_PER_GATE)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            run_program(st, one, 0, nat.SEM_SIMULATE, nat.EXEC_PER_GATE)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1) / reps
        name = "k_phase (cp, quarter of the state)"
        nbytes = 2 * 16 * (2 ** n) * 0.25
    achieved = nbytes / (ms * 1e-3) / 1e9
    traffic, tsrc = None, None
    if exec_mode == nat.EXEC_FUSED:
        traffic, tsrc = sweep_traffic(n)
    return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "bytes_per_launch": nbytes,
            "launch_ms": ms, "traffic": traffic, "traffic_source": tsrc}


def sweep_traffic(n: int):
    """DRAM bytes per sweep launch from the committed ncu capture, scaled to n qubits.

    The capture (26 qubits, 1 GiB state) is small enough for a full ncu set; a sweep's
    traffic scales with the 2^n amplitudes it streams."""
    f = ROOT / "profiles" / "k_sweep_qft26.md"
    try:
        for line in f.read_text().splitlines():
            if line.startswith("traffic_bytes_per_launch_at_26q"):
                b26 = float(line.split("=")[1])
                return b26 * 2.0 ** (n - 26), "ncu dram__bytes_read+write of k_sweep at 26 qubits x 2^(n-26)"
    except OSError:
        pass
    return None, None


def fused_sweep_timing(st, prog, stream, reps):
    """Average duration and algorithmic bytes of one fused sweep, from CUDA
    events around every sweep launch on the state's stream
    (dq_run_opts.time_sweeps).  Every sweep reads and writes the state
    (2 x 16 B per amplitude) except the first one after a reset, which
    generates its input from the basis index and only writes (16 B)."""
    from dqsim_bosonic_b200 import _native as nat
    from dqsim_bosonic_b200.statevector import run_program

    tot, cnt, runs = 0.0, 0, 0
    for _ in range(reps):
        st.reset()
        _, prof = run_program(st, prog, 7, nat.SEM_SIMULATE, nat.EXEC_FUSED, time_sweeps=True)
        tot += prof.sweep_time
        cnt += int(prof.sweeps)
        runs += 1 if prof.sweeps else 0
    n = prog.num_qubits
    nbytes = (2 * cnt - runs) * 16 * (2 ** n) / max(cnt, 1)
    return "k_sweep (fused tile sweep)", nbytes, tot / max(cnt, 1) * 1e3


if __name__ == "__main__":
    main()
