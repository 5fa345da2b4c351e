"""Module-level entry points and mode parsing.

Restates ``src/simulator.rs:13-113`` (``simulate_monolithic``,
``simulate_monolithic_shots``, ``simulate_distributed``,
``simulate_distributed_shots``) and ``src/codecs.rs:19-108`` (mode aliases,
option parsing and rejection, in the same order: the mode and options are
checked before the circuit is touched).

The ``state_vector`` and ``mps`` modes are backed by this engine (``mps``:
``dqsim_bosonic_b200.mps``).  The stabilizer and p-block backends of the
reference are not part of this build; selecting them parses the mode and
options exactly like the reference, reads the circuit, and then raises
``NotImplementedError``.
Distributed circuits run here by lowering them with
``as_monolithic_circuit()`` and simulating the result.
"""
from __future__ import annotations

from typing import Any

from .mps import MpsSimulator


def _ascii_lower(s: str) -> str:
    return "".join(chr(ord(c) + 32) if "A" <= c <= "Z" else c for c in s)


def _debug(s: str) -> str:
    return '"' + s.replace("\\", "\\\\").replace('"', '\\"') + '"'


def _norm_mode(mode: Any) -> str:
    if not isinstance(mode, str):
        raise TypeError(f"argument 'mode': expected str, got {type(mode).__name__}")
    return _ascii_lower(mode.strip()).replace("-", "_")


def parse_monolithic_mode(mode: Any) -> str:
    """``parse_monolithic_mode`` (codecs.rs:19-28)."""
    m = _norm_mode(mode)
    if m in ("state_vector", "statevector", "sv"):
        return "state_vector"
    if m in ("mps", "matrix_product_state"):
        return "mps"
    if m in ("stabilizer", "stab"):
        return "stabilizer"
    raise ValueError(
        f"Unsupported monolithic simulation mode {_debug(m)}; expected 'state_vector' or 'mps'"
    )


def parse_distributed_mode(mode: Any) -> str:
    """``parse_distributed_mode`` (codecs.rs:30-37)."""
    m = _norm_mode(mode)
    if m == "p_block":
        return "p_block"
    raise ValueError(f"Unsupported distributed simulation mode {_debug(m)}; expected 'p_block'")


def reject_monolithic_options(options: dict, mode: str) -> None:
    """``reject_monolithic_options`` (codecs.rs:68-84)."""
    if options:
        keys = "[" + ", ".join(_debug(k) for k in options) + "]"
        raise TypeError(f"Options {keys} are not supported for monolithic mode {_debug(mode)}")


def parse_mps_options(options: dict) -> tuple[int | None, float]:
    """``parse_mps_options`` (codecs.rs:39-66, 86-108)."""
    import math

    max_bond = None
    thr = 1e-12
    for key, value in options.items():
        if key == "max_bond_dimension":
            if value is None:
                max_bond = None
            else:
                if isinstance(value, bool) or not isinstance(value, int):
                    raise TypeError("max_bond_dimension must be an int or None")
                if value < 0:
                    raise OverflowError("can't convert negative int to unsigned")
                if value == 0:
                    raise ValueError("max_bond_dimension must be positive or None")
                max_bond = value
        elif key == "truncation_threshold":
            if isinstance(value, bool) or not isinstance(value, (int, float)):
                raise TypeError("truncation_threshold must be a float")
            v = float(value)
            if not math.isfinite(v) or v < 0.0:
                raise ValueError("truncation_threshold must be a finite non-negative float")
            thr = v
        else:
            raise TypeError(f"Unsupported MPS option {_debug(key)}")
    return max_bond, thr


def _out_of_scope(backend: str) -> NotImplementedError:
    return NotImplementedError(
        f"the {backend} backend is not part of the B200 statevector engine; "
        "use mode='state_vector' (distributed circuits: as_monolithic_circuit())"
    )


class StabilizerSimulator:
    """Placeholder for the reference's stabilizer backend (not built here)."""

    def __init__(self, seed=None):
        self.seed = seed

    def simulate_shots(self, circuit, shots=1000, profile=False):
        circuit.model_dump_json()
        raise _out_of_scope("stabilizer")


class PBlockSimulator:
    """Placeholder for the reference's p-block backend (not built here)."""

    def __init__(self, seed=None):
        self.seed = seed

    def simulate(self, distributed):
        raise _out_of_scope("p-block")

    def simulate_shots(self, distributed, shots=1000, profile=False):
        raise _out_of_scope("p-block")


class PBlockResult:
    """Placeholder for the reference's p-block result type (not built here)."""

    def __init__(self, *a, **k):
        raise _out_of_scope("p-block")


def simulate_monolithic(circuit, mode="state_vector", seed=None, profile=False, **options):
    """``simulate_monolithic`` (simulator.rs:13-45)."""
    from .statevector import StatevectorSimulator

    m = parse_monolithic_mode(mode)
    if m == "state_vector":
        reject_monolithic_options(options, mode)
        return StatevectorSimulator(seed, profile).simulate(circuit)
    if m == "mps":
        mb, thr = parse_mps_options(options)
        return MpsSimulator(seed, mb, thr).simulate(circuit)
    raise NotImplementedError(
        "Full statevector extraction ('simulate_monolithic') is not supported for stabilizer "
        "simulation. Please use shot-based sampling via 'simulate_monolithic_shots' instead."
    )


def simulate_monolithic_shots(circuit, mode="state_vector", shots=1000, seed=None, profile=False,
                              **options):
    """``simulate_monolithic_shots`` (simulator.rs:63-95)."""
    from .statevector import StatevectorSimulator

    m = parse_monolithic_mode(mode)
    if m == "state_vector":
        reject_monolithic_options(options, mode)
        return StatevectorSimulator(seed, False).simulate_shots(circuit, shots, profile)
    if m == "mps":
        mb, thr = parse_mps_options(options)
        return MpsSimulator(seed, mb, thr).simulate_shots(circuit, shots, profile)
    reject_monolithic_options(options, mode)
    return StabilizerSimulator(seed).simulate_shots(circuit, shots, profile)


def simulate_distributed(distributed, mode="p_block", seed=None):
    """``simulate_distributed`` (simulator.rs:47-61)."""
    parse_distributed_mode(mode)
    return PBlockSimulator(seed).simulate(distributed)


def simulate_distributed_shots(distributed, mode="p_block", shots=1000, seed=None, profile=False):
    """``simulate_distributed_shots`` (simulator.rs:97-113)."""
    parse_distributed_mode(mode)
    return PBlockSimulator(seed).simulate_shots(distributed, shots, profile)
