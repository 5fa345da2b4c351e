"""simulate_shots(profile=True) writes the reference's profile files (needs a B200).

Restates the statevector and MPS cases of the reference's tests/test_shots_profile.py
(dqsim package): no file without profile; with it exactly one
``dqsim_profiles/<backend>_shots_profile_*.json`` holding the common timing fields
(profiling.rs) and the backend's own (``fusion_time``; ``svd_calls``, ``svd_time``).
"""
import json

import pytest

from _circuits import JsonCircuit, g
from dqsim_bosonic_b200 import MpsSimulator, StatevectorSimulator

pytestmark = pytest.mark.gpu

SEED = 42


def _bell():
    return JsonCircuit(2, [g("h", 0), g("cx", 0, 1), g("measure", 0, 0), g("measure", 1, 1)], ncbits=2)


def _assert_common_fields(data, shots):
    assert data["num_shots"] == shots
    assert len(data["shot_times"]) == shots
    assert all(isinstance(t, float) and t >= 0.0 for t in data["shot_times"])
    for key in ("preprocessing_time", "shots_total_time", "total_time"):
        assert isinstance(data[key], float) and data[key] >= 0.0
    assert data["shots_total_time"] <= data["total_time"] + 1e-6


@pytest.mark.parametrize("sim_cls", [StatevectorSimulator, MpsSimulator])
def test_profile_false_does_not_write_file(sim_cls, tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    counts = sim_cls(seed=SEED).simulate_shots(_bell(), shots=50)
    assert sum(counts.values()) == 50
    assert set(counts) <= {"00", "11"}
    assert not (tmp_path / "dqsim_profiles").exists()


def test_statevector_profile_true_writes_json_file(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    counts = StatevectorSimulator(seed=SEED).simulate_shots(_bell(), shots=64, profile=True)
    assert sum(counts.values()) == 64
    files = list((tmp_path / "dqsim_profiles").glob("statevector_shots_profile_*.json"))
    assert len(files) == 1
    data = json.loads(files[0].read_text())
    _assert_common_fields(data, 64)
    assert isinstance(data["fusion_time"], float) and data["fusion_time"] >= 0.0


def test_mps_profile_true_writes_json_file(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    counts = MpsSimulator(seed=SEED).simulate_shots(_bell(), shots=64, profile=True)
    assert sum(counts.values()) == 64
    files = list((tmp_path / "dqsim_profiles").glob("mps_shots_profile_*.json"))
    assert len(files) == 1
    data = json.loads(files[0].read_text())
    _assert_common_fields(data, 64)
    assert isinstance(data["svd_calls"], int) and data["svd_calls"] > 0
    assert isinstance(data["svd_time"], float) and data["svd_time"] >= 0.0
