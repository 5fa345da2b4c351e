"""Batched trajectories on the GPU.

* :func:`run_trajectories` — many shots of one program (the ``simulate_shots``
  loop of statevector/simulator.rs:216-322): shot ``i`` starts from |0...0>
  with ``ChaCha8Rng::seed_from_u64(base_seed + i)`` (wrapping) under the shot
  semantics (fused single-qubit runs, ``run_instruction_par``).  Programs of up
  to 16 qubits run in ONE persistent launch of ``dq_run_trajectories`` (each
  trajectory held in the shared memory of a thread-block cluster); larger
  programs run shot by shot on the HBM engine (``dq_run``).
* :func:`run_batch` — a ragged batch of independent circuits, one trajectory
  each (``dq_run_batch``), optionally returning every final state.
* :class:`TrajectoryPlan` — a shot batch captured once as a CUDA graph and
  replayed with new seeds.
* :class:`TrajectoryTuner` — picks the launch geometry (threads per CTA,
  amplitudes per CTA, cluster span) by timing the candidates once per program
  shape.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _native as nat

_U64 = (1 << 64) - 1
MAX_RESIDENT_QUBITS = 16


def _opts(threads=0, max_cluster=0, local_bits=0) -> nat.TrajOpts:
    return nat.TrajOpts(int(threads), int(max_cluster), int(local_bits), 0)


def trajectories_resident(prog, base_seed: int, shots: int, device: int = 0, *, opts=None,
                          shot0: int = 0):
    """One persistent launch: returns (cbits[shots, cbit_space] int32, TrajStats)."""
    L = nat.lib()
    out = np.empty((shots, prog.cbit_space), dtype=np.int32)
    st = nat.TrajStats()
    o = opts if opts is not None else _opts()
    rc = L.dq_run_trajectories(int(device), prog.num_qubits, nat.ptr(prog.insts), prog.ninst,
                               nat.ptr(prog.conds) if prog.conds.size else None, prog.conds.size,
                               base_seed & _U64, int(shot0), int(shots),
                               nat.ptr(out) if out.size else None, prog.cbit_space,
                               ctypes.byref(o), ctypes.byref(st))
    _check_traj(rc, prog, st, "dq_run_trajectories")
    return out, st


def _check_traj(rc: int, prog, st, what: str) -> None:
    """Unsupported generic gates surface as the shot path's RuntimeError
    with the reference's message; other failures as in nat.check."""
    if rc == nat.DQ_ERR_UNSUPPORTED and st.failed_inst >= 0:
        from .statevector import _unsupported_message

        raise RuntimeError(_unsupported_message(prog, st.failed_inst & ((1 << 40) - 1)))
    nat.check(rc, what)


def run_trajectories(prog, base_seed: int, shots: int, device: int, want_times: bool = False,
                     *, tuner=None):
    """Returns (cbits[shots, cbit_space] int32, per-shot seconds, fusion seconds).

    ``tuner``: a :class:`TrajectoryTuner`, ``False`` for the default geometry,
    or ``None`` (tune batches of 4096 shots or more).

    Resident launches report the launch's device time spread evenly over its
    shots (the shots run concurrently); fusion seconds are the engine's host
    time fusing and encoding the program."""
    if shots and prog.num_qubits <= MAX_RESIDENT_QUBITS:
        if tuner is None and shots >= 4096:
            tuner = default_tuner()
        o = tuner.choose(prog, device) if tuner else _opts()
        out, st = trajectories_resident(prog, base_seed, shots, device, opts=o)
        per = st.kernel_ms * 1e-3 / shots
        return out, ([per] * shots if want_times else []), st.prepare_ms * 1e-3
    from .statevector import run_program

    state = nat.State(prog.num_qubits, device)
    out = np.empty((shots, prog.cbit_space), dtype=np.int32)
    times: list[float] = []
    for i in range(shots):
        t0 = time.perf_counter()
        if i:
            state.reset()
        cbits, _ = run_program(state, prog, (base_seed + i) & _U64, nat.SEM_SHOTS, nat.EXEC_FUSED)
        out[i] = cbits
        if want_times:
            times.append(time.perf_counter() - t0)
    state.release()
    return out, times, 0.0


def run_batch(progs, seeds, device: int = 0, *, want_states=False, opts=None):
    """Independent circuits, one trajectory each (shot semantics), in one
    persistent launch (``dq_run_batch``).

    ``want_states``: True for every item's final state, or a collection of
    item indices to return the states of those items only.
    Returns (list of cbits arrays, list of final states (None where not
    requested) or None, TrajStats)."""
    progs = list(progs)
    seeds = [int(s) & _U64 for s in seeds]
    if len(seeds) != len(progs):
        raise ValueError("one seed per program")
    items = (nat.BatchItem * max(1, len(progs)))()
    cbits = []
    states = []
    pick = None if isinstance(want_states, bool) else set(int(i) for i in want_states)
    for k, (p, s) in enumerate(zip(progs, seeds)):
        cb = np.full(p.cbit_space, -1, dtype=np.int32)
        wanted = (k in pick) if pick is not None else bool(want_states)
        sv = np.empty(1 << p.num_qubits, dtype=np.complex128) if wanted else None
        cbits.append(cb)
        states.append(sv)
        it = items[k]
        it.n = p.num_qubits
        it.prog = nat.ptr(p.insts)
        it.ninst = p.ninst
        it.conds = nat.ptr(p.conds) if p.conds.size else None
        it.nconds = p.conds.size
        it.seed = s
        it.cbits_out = nat.ptr(cb) if cb.size else None
        it.ncbits = cb.size
        it.state_out = nat.ptr(sv) if sv is not None else None
    st = nat.TrajStats()
    o = opts if opts is not None else _opts()
    rc = nat.lib().dq_run_batch(int(device), ctypes.addressof(items), len(progs),
                                ctypes.byref(o), ctypes.byref(st))
    if rc == nat.DQ_ERR_UNSUPPORTED and st.failed_inst >= 0:
        from .statevector import _unsupported_message

        k = st.failed_inst >> 40
        raise RuntimeError(f"batch item {k}: " +
                           _unsupported_message(progs[k], st.failed_inst & ((1 << 40) - 1)))
    nat.check(rc, "dq_run_batch")
    return cbits, (states if (pick is not None or want_states) else None), st


class TrajectoryPlan:
    """A shot batch of one program captured as a CUDA graph and replayed.

    ``run(base_seed)`` replays the graph (seed upload, counter reset, the
    persistent launch, result copies) and returns (cbits, TrajStats) for shots
    ``base_seed + s``, s < shots."""

    def __init__(self, prog, shots: int, device: int = 0, *, opts=None):
        self.prog = prog
        self.shots = int(shots)
        self.device = int(device)
        h = ctypes.c_void_p()
        o = opts if opts is not None else _opts()
        nat.check(nat.lib().dq_traj_plan_create(
            self.device, prog.num_qubits, nat.ptr(prog.insts), prog.ninst,
            nat.ptr(prog.conds) if prog.conds.size else None, prog.conds.size, self.shots,
            prog.cbit_space, ctypes.byref(o), ctypes.byref(h)), "dq_traj_plan_create")
        self._h = h

    def run(self, base_seed: int):
        if self._h is None:
            raise ValueError("plan was released")
        out = np.empty((self.shots, self.prog.cbit_space), dtype=np.int32)
        st = nat.TrajStats()
        rc = nat.lib().dq_traj_plan_run(self._h, base_seed & _U64,
                                        nat.ptr(out) if out.size else None, ctypes.byref(st))
        _check_traj(rc, self.prog, st, "dq_traj_plan_run")
        return out, st

    def release(self) -> None:
        if getattr(self, "_h", None) is not None:
            nat.lib().dq_traj_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class TrajectoryTuner:
    """Chooses threads per CTA and amplitudes per CTA for resident trajectories.

    For a program shape (qubits, instruction count) it times each candidate
    geometry once on a short batch (the real program, seeds offset far from
    the caller's) and keeps the fastest; later calls reuse the choice."""

    def __init__(self, trial_shots: int = 256):
        self.trial_shots = int(trial_shots)
        self.cache: dict[tuple, nat.TrajOpts] = {}
        self.timings: dict[tuple, list] = {}

    @staticmethod
    def candidates(n: int):
        out = []
        for threads in (128, 256, 512):
            lbs = {min(n, 13)}
            if n > 11:
                lbs.add(n - 1 if n <= 14 else 13)
            for lb in sorted(lbs):
                if n - lb <= 3:
                    out.append(_opts(threads, 8, lb))
        return out

    def choose(self, prog, device: int = 0) -> nat.TrajOpts:
        key = (prog.num_qubits, prog.ninst, device)
        if key in self.cache:
            return self.cache[key]
        best, best_ms, rows = None, float("inf"), []
        for o in self.candidates(prog.num_qubits):
            try:
                _, st = trajectories_resident(prog, 0x5EED_0000_0000, self.trial_shots, device, opts=o)
            except (ValueError, nat.EngineError):
                continue
            rows.append((o.threads, o.local_bits, st.cluster_span, st.kernel_ms))
            if st.kernel_ms < best_ms:
                best, best_ms = o, st.kernel_ms
        if best is None:
            best = _opts()
        self.cache[key] = best
        self.timings[key] = rows
        return best


_default_tuner: TrajectoryTuner | None = None


def default_tuner() -> TrajectoryTuner:
    global _default_tuner
    if _default_tuner is None:
        _default_tuner = TrajectoryTuner()
    return _default_tuner
