"""B200-native FP64 statevector engine with the Python API of ``dqsim``.

Same exported names as the reference package (``dqsim/__init__.py``); the
statevector classes and ``state_vector`` mode run on hand-written sm_100a
CUDA kernels through the C ABI of ``include/dqsim_cuda.h``.
"""
from .simulator import (
    MpsSimulator,
    PBlockResult,
    PBlockSimulator,
    StabilizerSimulator,
    simulate_distributed,
    simulate_distributed_shots,
    simulate_monolithic,
    simulate_monolithic_shots,
)
from .statevector import SimulationProfile, SimulationResult, StatevectorSimulator

__all__ = [
    "StatevectorSimulator",
    "StabilizerSimulator",
    "MpsSimulator",
    "SimulationResult",
    "SimulationProfile",
    "PBlockSimulator",
    "PBlockResult",
    "simulate_monolithic",
    "simulate_distributed",
    "simulate_monolithic_shots",
    "simulate_distributed_shots",
]
