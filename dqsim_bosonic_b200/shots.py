"""``simulate_shots``: independent per-shot trajectories.

Restates ``StatevectorSimulator::simulate_shots``
(src/monolithic/statevector/simulator.rs:216-322): the circuit is fused once
(``fuse_circuit``, types.rs:248-293, done inside the engine), shot ``i``
starts from |0...0> with ``ChaCha8Rng::seed_from_u64(base_seed + i)``
(wrapping), and each shot's classical register is formatted MSB-first and
counted.  With ``profile=True`` a JSON profile is written to
``./dqsim_profiles/statevector_shots_profile_<unix_ns>.json`` (profiling.rs).
"""
from __future__ import annotations

import json
import os
import time
from pathlib import Path

import numpy as np

from . import _native as nat
from .circuit import format_cbits

_U64 = (1 << 64) - 1


def write_shots_profile(prefix: str, profile: dict) -> Path:
    """``write_shots_profile`` (src/profiling.rs:8-18)."""
    d = Path("dqsim_profiles")
    d.mkdir(parents=True, exist_ok=True)
    path = d / f"{prefix}_shots_profile_{time.time_ns()}.json"
    path.write_text(json.dumps(profile, indent=2))
    return path


def run_shots(sim, circuit, shots: int, profile: bool) -> dict[str, int]:
    from .statevector import _entropy_u64, _parse, run_program

    total_t0 = time.perf_counter()
    prog, prep = _parse(circuit)
    base_seed = sim._seed if sim._seed is not None else _entropy_u64()
    counts: dict[str, int] = {}
    shot_times: list[float] = []
    shots_t0 = time.perf_counter()
    fusion_time = 0.0
    if shots:
        from .batch import run_trajectories

        bits, shot_times, fusion_time = run_trajectories(prog, base_seed, shots, sim.device,
                                                         want_times=profile)
        keys = [format_cbits(row, prog.num_cbits) for row in bits]
        for k in keys:
            counts[k] = counts.get(k, 0) + 1
    shots_total = time.perf_counter() - shots_t0
    if profile:
        write_shots_profile(
            "statevector",
            {
                "preprocessing_time": prep,
                "fusion_time": fusion_time,
                "shots_total_time": shots_total,
                "total_time": time.perf_counter() - total_t0,
                "num_shots": shots,
                "shot_times": [float(t) for t in shot_times],
            },
        )
    return counts
