"""Batched trajectories: many shots of one circuit on the GPU.

``run_trajectories`` runs shot ``i`` of a program with the seed
``base_seed + i`` (wrapping) under the shots semantics of the reference
(fused single-qubit runs, ``run_instruction_par``) and returns each shot's
classical register.
"""
from __future__ import annotations

import time

import numpy as np

from . import _native as nat

_U64 = (1 << 64) - 1


def run_trajectories(prog, base_seed: int, shots: int, device: int, want_times: bool = False):
    """Returns (cbits[shots, cbit_space] int32, per-shot seconds, fusion seconds)."""
    from .statevector import run_program

    state = nat.State(prog.num_qubits, device)
    out = np.empty((shots, prog.cbit_space), dtype=np.int32)
    times: list[float] = []
    for i in range(shots):
        t0 = time.perf_counter()
        if i:
            state.reset()
        cbits, _ = run_program(state, prog, (base_seed + i) & _U64, nat.SEM_SHOTS, nat.EXEC_PER_GATE)
        out[i] = cbits
        if want_times:
            times.append(time.perf_counter() - t0)
    state.release()
    return out, times, 0.0
