"""``MpsSimulator`` on the device (src/monolithic/mps/simulator.rs:293-455).

The matrix-product state lives in HBM behind a ``dq_mps_t`` handle; every
gate, measurement and reset of the program runs as a kernel over the batch
of states (one CTA per state), two-qubit gates as fused contract / SVD /
truncate / split steps.  ``simulate`` returns the same ``SimulationResult``
as the statevector backend: the MPS is contracted into a device statevector
(to_statevector, :238-257) that the result's queries read.
``simulate_shots`` runs the shots as one batch of independent MPS per launch.
"""
from __future__ import annotations

import ctypes
import time
from typing import Any

import numpy as np

from . import _native as nat
from .circuit import Program, format_cbits

_U64 = (1 << 64) - 1
_MULTI = ("MPS simulator only supports one- and two-qubit unitary gates plus measurement, "
          "reset, and conditionals")


def _check_opt_usize(v: Any, what: str) -> int | None:
    if v is None:
        return None
    if isinstance(v, bool) or not isinstance(v, int):
        raise TypeError(f"argument '{what}': expected int or None, got {type(v).__name__}")
    if v < 0:
        raise OverflowError("can't convert negative int to unsigned")
    if v >= (1 << 64):
        raise OverflowError("int too big to convert")
    return int(v)


def _check_f64(v: Any, what: str) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise TypeError(f"argument '{what}': must be real number, not {type(v).__name__}")
    return float(v)


def _unsupported(prog: Program, failed: int) -> NotImplementedError:
    """The dispatcher's two rejections (simulator.rs:540-557)."""
    from .statevector import _rust_debug_str

    rec = prog.insts[int(failed)] if 0 <= int(failed) < prog.ninst else None
    if rec is not None and int(rec["kind"]) == nat.KIND["g_unsupported"]:
        name = prog.gate_names.get(int(failed), "?")
        return NotImplementedError(f"MPS simulator does not support generic gate {_rust_debug_str(name)}")
    return NotImplementedError(_MULTI)


def _bond_arg(max_bond: int | None) -> int:
    if max_bond is None:
        return 0
    return min(max(int(max_bond), 1), (1 << 31))


class MpsHandle:
    """Owning wrapper of one device MPS (``dq_mps_t``)."""

    def __init__(self, n: int, device: int, max_bond: int | None, threshold: float):
        h = ctypes.c_void_p()
        nat.check(nat.lib().dq_mps_create(int(n), int(device), _bond_arg(max_bond), float(threshold),
                                          ctypes.byref(h)), "dq_mps_create")
        self._h = h
        self.n = int(n)
        self.device = int(device)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("MPS was released")
        return self._h

    def release(self) -> None:
        if getattr(self, "_h", None) is not None:
            nat.lib().dq_mps_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def run(self, prog: Program, seed: int) -> tuple[np.ndarray, nat.MpsStats]:
        cbits = np.full(prog.cbit_space, -1, dtype=np.int32)
        st = nat.MpsStats()
        rc = nat.lib().dq_mps_run(self.handle, nat.ptr(prog.insts), prog.ninst,
                                  nat.ptr(prog.conds) if prog.conds.size else None,
                                  prog.conds.shape[0], seed & _U64, nat.ptr(cbits), cbits.size,
                                  ctypes.byref(st))
        if rc == nat.DQ_ERR_UNSUPPORTED:
            raise _unsupported(prog, st.failed_inst)
        nat.check(rc, "dq_mps_run")
        return cbits, st

    def apply_2q(self, a: int, b: int, u: np.ndarray) -> None:
        m = np.ascontiguousarray(np.asarray(u, dtype=np.complex128).reshape(4, 4))
        nat.check(nat.lib().dq_mps_apply_2q(self.handle, int(a), int(b), nat.ptr(m)), "dq_mps_apply_2q")

    def reserve(self, capacity: int) -> None:
        nat.check(nat.lib().dq_mps_reserve(self.handle, int(capacity)), "dq_mps_reserve")

    def bond_dims(self) -> list[int]:
        d = np.zeros(self.n + 1, dtype=np.uint32)
        nat.check(nat.lib().dq_mps_bond_dims(self.handle, nat.ptr(d)), "dq_mps_bond_dims")
        return [int(x) for x in d]

    def to_state(self) -> nat.State:
        st = nat.State(self.n, self.device)
        nat.check(nat.lib().dq_mps_to_state(self.handle, st.handle), "dq_mps_to_state")
        return st


def run_mps_shots(prog: Program, base_seed: int, shots: int, device: int, max_bond: int | None,
                  threshold: float, batch: int = 0) -> tuple[np.ndarray, nat.MpsStats]:
    """cbits of ``shots`` MPS trajectories (row i seeded base_seed + i)."""
    cb = np.full((max(shots, 0), prog.cbit_space), -1, dtype=np.int32)
    st = nat.MpsStats()
    rc = nat.lib().dq_mps_run_shots(int(device), prog.num_qubits, _bond_arg(max_bond), float(threshold),
                                    nat.ptr(prog.insts), prog.ninst,
                                    nat.ptr(prog.conds) if prog.conds.size else None,
                                    prog.conds.shape[0], base_seed & _U64, 0, int(shots),
                                    nat.ptr(cb) if cb.size else None, prog.cbit_space, int(batch),
                                    ctypes.byref(st))
    if rc == nat.DQ_ERR_UNSUPPORTED:
        raise _unsupported(prog, st.failed_inst)
    nat.check(rc, "dq_mps_run_shots")
    return cb, st


class MpsSimulator:
    """Matrix-product-state simulator (simulator.rs:293-455) on one B200.

    ``max_bond_dimension`` caps every bond (None: no cap); singular values at
    or below ``truncation_threshold`` are dropped (at least one is kept) and
    the kept ones are rescaled to the full norm.  Keyword extension:
    ``device`` (CUDA ordinal).
    """

    def __init__(self, seed=None, max_bond_dimension=None, truncation_threshold=1e-12, *,
                 device: int | None = None):
        from .statevector import _check_u64, _default_device

        self._seed = None if seed is None else _check_u64(seed, "seed")
        self._max_bond = _check_opt_usize(max_bond_dimension, "max_bond_dimension")
        self._threshold = _check_f64(truncation_threshold, "truncation_threshold")
        self.device = _default_device() if device is None else int(device)

    def simulate(self, circuit):
        """Run the circuit on one MPS and return a ``SimulationResult``."""
        from .statevector import SimulationResult, _entropy_u64, _parse

        prog, _ = _parse(circuit)
        seed = self._seed if self._seed is not None else _entropy_u64()
        n = prog.num_qubits
        if n == 0:
            return _empty_result(self.device)
        mps = MpsHandle(n, self.device, self._max_bond, self._threshold)
        try:
            cbits, _ = mps.run(prog, seed)
            state = mps.to_state()
        finally:
            mps.release()
        cb = {i: int(v) for i, v in enumerate(cbits.tolist()) if v >= 0}
        return SimulationResult(state, n, cb, None)

    def simulate_shots(self, circuit, shots=1000, profile=False) -> dict[str, int]:
        """``shots`` independent MPS trajectories; returns bitstring counts."""
        from .shots import write_shots_profile
        from .statevector import _check_u64, _entropy_u64, _parse

        shots = _check_u64(shots, "shots")
        total_t0 = time.perf_counter()
        prog, prep = _parse(circuit)
        base_seed = self._seed if self._seed is not None else _entropy_u64()
        counts: dict[str, int] = {}
        shots_t0 = time.perf_counter()
        svd_calls, svd_time = 0, 0.0
        if shots:
            if prog.num_qubits == 0:
                bits = np.full((shots, prog.cbit_space), -1, dtype=np.int32)
            else:
                bits, st = run_mps_shots(prog, base_seed, shots, self.device, self._max_bond,
                                         self._threshold)
                svd_calls, svd_time = int(st.svd_calls), float(st.kernel_ms) / 1e3
            for row in bits:
                k = format_cbits(row, prog.num_cbits)
                counts[k] = counts.get(k, 0) + 1
        shots_total = time.perf_counter() - shots_t0
        if profile:
            write_shots_profile(
                "mps",
                {
                    "preprocessing_time": prep,
                    "shots_total_time": shots_total,
                    "total_time": time.perf_counter() - total_t0,
                    "num_shots": shots,
                    "shot_times": [shots_total / shots] * shots if shots else [],
                    "svd_calls": svd_calls,
                    "svd_time": svd_time,
                },
            )
        return counts


def _empty_result(device: int):
    """A zero-qubit circuit: the statevector is [1] (Mps::new(0).to_statevector())."""
    from .statevector import SimulationResult

    state = nat.State(0, device)
    return SimulationResult(state, 0, {}, None)
