"""``StatevectorSimulator`` / ``SimulationResult`` / ``SimulationProfile``.

Python restatement of the PyO3 classes of
``src/monolithic/statevector/simulator.rs`` (same constructor keywords,
methods, return types and exception types) on top of the C ABI: the state
vector stays in HBM inside a ``dq_state_t`` handle, and every gate, measure
and query runs as a CUDA kernel for sm_100a.
"""
from __future__ import annotations

import ctypes
import json
import os
import time
from pathlib import Path
from typing import Any

import numpy as np

from . import _native as nat
from .circuit import CircuitDecodeError, Program, circuit_json, decode_program, format_cbits

_U64 = (1 << 64) - 1


def _default_device() -> int:
    env = os.environ.get("DQSIM_DEVICE")
    if env is not None:
        return int(env)
    return int(os.environ.get("LOCAL_RANK", "0"))


def _default_exec() -> int:
    mode = os.environ.get("DQSIM_EXEC", "fused").strip().lower()
    return nat.EXEC_PER_GATE if mode in ("per_gate", "per-gate", "exact") else nat.EXEC_FUSED


def _check_u64(v: Any, what: str) -> int:
    if isinstance(v, bool) or not isinstance(v, int):
        raise TypeError(f"argument '{what}': expected an unsigned 64-bit int, got {type(v).__name__}")
    if v < 0 or v > _U64:
        raise OverflowError(f"argument '{what}': {v} does not fit an unsigned 64-bit int")
    return v


def _entropy_u64() -> int:
    return int.from_bytes(os.urandom(8), "little")


def _rust_debug_str(s: str) -> str:
    return '"' + s.replace("\\", "\\\\").replace('"', '\\"') + '"'


class SimulationProfile:
    """Per-kernel-class call counts and times (simulator.rs:52-88)."""

    __slots__ = (
        "apply_one_qubit_calls",
        "apply_one_qubit_time",
        "apply_n_qubit_calls",
        "apply_n_qubit_time",
        "measure_qubit_calls",
        "measure_qubit_time",
        "total_time",
        "kernel_launches",
        "sweeps",
        "boundary_draws",
    )

    def __init__(self, p: nat.Profile):
        for name in self.__slots__:
            setattr(self, name, getattr(p, name))

    def __repr__(self) -> str:
        total = max(self.total_time, 1e-9)
        return (
            f"SimulationProfile (total: {self.total_time * 1000.0:.2f} ms)\n"
            f"  apply_one_qubit : {self.apply_one_qubit_calls:4} calls  "
            f"{self.apply_one_qubit_time * 1000.0:8.2f} ms  ({100.0 * self.apply_one_qubit_time / total:.1f}%)\n"
            f"  apply_n_qubit   : {self.apply_n_qubit_calls:4} calls  "
            f"{self.apply_n_qubit_time * 1000.0:8.2f} ms  ({100.0 * self.apply_n_qubit_time / total:.1f}%)\n"
            f"  measure_qubit   : {self.measure_qubit_calls:4} calls  "
            f"{self.measure_qubit_time * 1000.0:8.2f} ms  ({100.0 * self.measure_qubit_time / total:.1f}%)"
        )


def _check_marginal_qubits(qubits, n: int) -> list[int]:
    if qubits is None:
        return list(range(n - 1, -1, -1))
    qs = []
    for q in qubits:
        qs.append(_check_u64(q, "qubits"))
    for q in qs:
        if q >= n:
            raise ValueError(f"qubit {q} out of range for a {n}-qubit state")
    if len(set(qs)) != len(qs):
        raise ValueError("repeated qubit in the qubit list")
    if len(qs) > 30:
        raise ValueError("at most 30 qubits per marginal distribution")
    return qs


class SimulationResult:
    """Final state and classical bits of one ``simulate`` call (simulator.rs:94-192)."""

    def __init__(self, state: nat.State, num_qubits: int, cbits: dict[int, int],
                 profile: SimulationProfile | None):
        self._state = state
        self.num_qubits = num_qubits
        self._cbits = cbits
        self._profile = profile
        self.last_boundary_draws = 0
        # host-side phase times (ms) of the call that made this result and of
        # its latest probability query: parse, state, run, engine, query
        self.timings: dict[str, float] = {}

    @property
    def statevector(self) -> np.ndarray:
        """Raw complex amplitudes as a NumPy array of shape (2^n,) (a copy)."""
        return self._state.download()

    @property
    def classical_bits(self) -> dict[int, int]:
        return dict(self._cbits)

    @property
    def profile(self) -> SimulationProfile | None:
        return self._profile

    @property
    def state_handle(self) -> nat.State:
        """The device-resident state (for zero-copy consumers)."""
        return self._state

    def _marginal(self, qs: list[int]) -> np.ndarray:
        t0 = time.perf_counter()
        out = np.empty(1 << len(qs), dtype=np.float64)
        q = np.asarray(qs, dtype=np.uint32)
        nat.check(nat.lib().dq_marginal_probs(self._state.handle, nat.ptr(q), len(qs), nat.ptr(out)),
                  "dq_marginal_probs")
        self.timings["query_ms"] = (time.perf_counter() - t0) * 1e3
        return out

    def probability_array(self, qubits=None) -> np.ndarray:
        """Marginal distribution as a dense float64 array (index j, qubits[0] = MSB)."""
        return self._marginal(_check_marginal_qubits(qubits, self.num_qubits))

    def probabilities(self, qubits=None) -> dict[int, float]:
        """Full or marginal distribution; keys are basis-state ints, p > 0 only."""
        probs = self.probability_array(qubits)
        nz = np.flatnonzero(probs > 0.0)
        return dict(zip(nz.tolist(), probs[nz].tolist()))

    def sample_indices(self, shots: int = 1000, qubits=None, seed=None) -> np.ndarray:
        """Per-shot sampled indices (device CDF + device ChaCha8 draws)."""
        shots = _check_u64(shots, "shots")
        qs = _check_marginal_qubits(qubits, self.num_qubits)
        out = np.empty(max(shots, 1), dtype=np.uint32)
        q = np.asarray(qs, dtype=np.uint32)
        nb = ctypes.c_uint64(0)
        L = nat.lib()
        if seed is None:
            key = np.frombuffer(os.urandom(32), dtype=np.uint32).copy()
            rc = L.dq_sample_key(self._state.handle, nat.ptr(q), len(qs), nat.ptr(key), shots,
                                 nat.ptr(out), ctypes.byref(nb))
        else:
            rc = L.dq_sample(self._state.handle, nat.ptr(q), len(qs), _check_u64(seed, "seed"), shots,
                             nat.ptr(out), ctypes.byref(nb))
        nat.check(rc, "dq_sample")
        self.last_boundary_draws = int(nb.value)
        return out[:shots]

    def counts(self, shots: int = 1000, qubits=None, seed=None) -> dict[str, int]:
        """Sampled bitstring counts; qubits[0] is the leftmost character."""
        idx = self.sample_indices(shots, qubits, seed)
        k = self.num_qubits if qubits is None else len(list(qubits))
        if idx.size == 0:
            return {}
        vals, cnt = np.unique(idx, return_counts=True)
        return {format(int(v), f"0{k}b"): int(c) for v, c in zip(vals, cnt)}

    def fidelity(self, other) -> float:
        """|<self|other>|^2; 0.0 when the lengths differ (simulator.rs:184-191)."""
        if not isinstance(other, np.ndarray) or other.dtype != np.complex128 or other.ndim != 1:
            raise TypeError("fidelity() expects a 1-D numpy.ndarray of complex128")
        if other.shape[0] != (1 << self.num_qubits):
            return 0.0
        a = np.ascontiguousarray(other)
        re, im = ctypes.c_double(0.0), ctypes.c_double(0.0)
        nat.check(nat.lib().dq_inner(self._state.handle, nat.ptr(a), a.shape[0], ctypes.byref(re),
                                     ctypes.byref(im)), "dq_inner")
        return re.value * re.value + im.value * im.value


def _parse(circuit: Any) -> tuple[Program, float]:
    t0 = time.perf_counter()
    text = circuit_json(circuit)
    try:
        prog = decode_program(text)
    except CircuitDecodeError as e:
        raise ValueError(f"Circuit JSON parse error: {e}") from None
    return prog, time.perf_counter() - t0


def _unsupported_message(prog: Program, failed: int) -> str:
    name = prog.gate_names.get(int(failed), "?")
    return f"Unsupported generic gate: {_rust_debug_str(name)}. Decompose it before simulating."


def run_program(state: nat.State, prog: Program, seed: int, semantics: int, exec_mode: int,
                fusion_width: int = 0, profile: bool = False, time_sweeps: bool = False,
                max_cost: int = 0) -> tuple[np.ndarray, nat.Profile]:
    """One ``dq_run`` over ``prog``; returns (cbits array, engine profile)."""
    cbits = np.full(prog.cbit_space, -1, dtype=np.int32)
    opts = nat.RunOpts(semantics, exec_mode, fusion_width, 1 if profile else 0,
                       1 if time_sweeps else 0, int(max_cost))
    prof = nat.Profile()
    rc = nat.lib().dq_run(state.handle, nat.ptr(prog.insts), prog.ninst,
                          nat.ptr(prog.conds) if prog.conds.size else None, prog.conds.shape[0],
                          seed & _U64, nat.ptr(cbits), cbits.size, ctypes.byref(opts), ctypes.byref(prof))
    if rc == nat.DQ_ERR_UNSUPPORTED:
        msg = _unsupported_message(prog, prof.failed_inst)
        if semantics == nat.SEM_SHOTS:
            raise RuntimeError(msg)
        raise NotImplementedError(msg)
    nat.check(rc, "dq_run")
    return cbits, prof


class StatevectorSimulator:
    """FP64 statevector simulator on one B200 (simulator.rs:198-380).

    Keyword extensions beyond the reference: ``device`` (CUDA ordinal),
    ``exec`` ("fused" tile sweeps or "per_gate" exact kernels) and
    ``fusion_width`` (local qubits per fused tile, 0 = engine default).
    """

    def __init__(self, seed=None, profile=False, *, device: int | None = None,
                 exec: str | None = None, fusion_width: int = 0):
        self._seed = None if seed is None else _check_u64(seed, "seed")
        self._profile = bool(profile)
        self.device = _default_device() if device is None else int(device)
        if exec is None:
            self._exec = _default_exec()
        else:
            e = exec.strip().lower().replace("-", "_")
            if e not in ("fused", "per_gate"):
                raise ValueError("exec must be 'fused' or 'per_gate'")
            self._exec = nat.EXEC_FUSED if e == "fused" else nat.EXEC_PER_GATE
        self.fusion_width = int(fusion_width)

    def simulate(self, circuit) -> SimulationResult:
        """Run the circuit and return a ``SimulationResult``."""
        prog, parse_s = _parse(circuit)
        seed = self._seed if self._seed is not None else _entropy_u64()
        t0 = time.perf_counter()
        state = nat.State(prog.num_qubits, self.device)
        t1 = time.perf_counter()
        exec_mode = nat.EXEC_PER_GATE if self._profile else self._exec
        cbits, prof = run_program(state, prog, seed, nat.SEM_SIMULATE, exec_mode, self.fusion_width,
                                  self._profile)
        t2 = time.perf_counter()
        cb = {i: int(v) for i, v in enumerate(cbits.tolist()) if v >= 0}
        res = SimulationResult(state, prog.num_qubits, cb,
                               SimulationProfile(prof) if self._profile else None)
        res.last_boundary_draws = int(prof.boundary_draws)
        # run_ms: the dq_run call (it returns once the state is final);
        # engine_ms: the engine's own clock inside that call
        res.timings = {"parse_ms": parse_s * 1e3, "state_ms": (t1 - t0) * 1e3,
                       "run_ms": (t2 - t1) * 1e3, "engine_ms": float(prof.total_time) * 1e3}
        return res

    def simulate_shots(self, circuit, shots=1000, profile=False) -> dict[str, int]:
        """Run ``shots`` independent trajectories; returns bitstring counts."""
        from .shots import run_shots

        return run_shots(self, circuit, _check_u64(shots, "shots"), bool(profile))
