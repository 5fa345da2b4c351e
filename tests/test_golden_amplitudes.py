"""Amplitude-level golden fixtures (tests/golden/amp_*.json).

The fixtures hold closed-form final statevectors of small circuits written
from the gate definitions of src/gates.rs (tests/golden/make_amplitudes.py),
so they pin the phase conventions a probability cannot see: the sign of
rz / crz / rzz angles, u3's phase placement, qubits[0] as the most
significant bit of a gate index, the Bell states of the remote-link gates,
and the full QFT phase ladder.  The oracle is checked against them on the
CPU; the engine (per-gate kernels and fused tile sweeps) on the GPU.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import _oracle
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURES = sorted(GOLDEN.glob("amp_*.json"))


def load(path):
    d = json.loads(path.read_text())
    want = np.array([complex(a, b) for a, b in d["amplitudes"]])
    prog = encode(decode_circuit_json(json.dumps(d["circuit"])))
    return d, prog, want


def test_fixture_set_is_complete():
    names = {p.stem for p in FIXTURES}
    for must in ("amp_rz_plus", "amp_u3_one", "amp_cp_plus", "amp_crz_plus", "amp_rzz_plus",
                 "amp_psi_plus_bell", "amp_psi_minus_bell", "amp_qft8_basis_229"):
        assert must in names
    assert len(FIXTURES) >= 30


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.stem)
def test_oracle_matches_closed_form(path):
    d, prog, want = load(path)
    got, _, rc, _ = _oracle.run(prog, 1)
    assert rc == 0
    assert np.max(np.abs(got - want)) <= d["atol"]


def _flip_angles(circ):
    out = json.loads(json.dumps(circ))
    for ins in out["instructions"]:
        for k in ("theta", "phi", "lam", "gamma"):
            if k in ins:
                ins[k] = -ins[k]
    return out


@pytest.mark.parametrize("name", ["amp_rz_plus", "amp_crz_plus", "amp_rzz_plus", "amp_cp_plus",
                                  "amp_u3_one", "amp_cu_gamma", "amp_rxx_zero"])
def test_fixtures_see_the_sign_of_an_angle(name):
    """A planted sign error (every angle negated) on the oracle's input must
    fail the fixture: the pins are not satisfied by the conjugate convention."""
    d = json.loads((GOLDEN / f"{name}.json").read_text())
    want = np.array([complex(a, b) for a, b in d["amplitudes"]])
    prog = encode(decode_circuit_json(json.dumps(_flip_angles(d["circuit"]))))
    got, _, rc, _ = _oracle.run(prog, 1)
    assert rc == 0
    assert np.max(np.abs(got - want)) > 1e-3


def test_fixtures_see_psi_plus_against_psi_minus():
    d = json.loads((GOLDEN / "amp_psi_plus_bell.json").read_text())
    want = np.array([complex(a, b) for a, b in d["amplitudes"]])
    circ = json.loads(json.dumps(d["circuit"]))
    circ["instructions"][0]["name"] = "remote_link_psi_minus"
    got, _, _, _ = _oracle.run(encode(decode_circuit_json(json.dumps(circ))), 1)
    assert np.max(np.abs(got - want)) > 0.5


def test_qft_closed_form_matches_generator():
    """amp[w] = exp(2 pi i rev(x) rev(w) / 2^n) / 2^(n/2) for the QFT of |x>."""
    d, _, want = load(GOLDEN / "amp_qft5_basis_22.json")
    n, x = 5, 0b10110
    rev = lambda v: int(format(v, f"0{n}b")[::-1], 2)
    for w in range(1 << n):
        ph = 2 * math.pi * ((rev(x) * rev(w)) % (1 << n)) / (1 << n)
        assert abs(want[w] - complex(math.cos(ph), math.sin(ph)) / math.sqrt(1 << n)) < 1e-15


@pytest.mark.gpu
@pytest.mark.parametrize("exec_mode", ["per_gate", "fused"])
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: p.stem)
def test_engine_matches_closed_form(gpu, path, exec_mode):
    from dqsim_bosonic_b200 import StatevectorSimulator

    d, _, want = load(path)

    class C:
        def model_dump_json(self):
            return json.dumps(d["circuit"])

    res = StatevectorSimulator(seed=1, device=0, exec=exec_mode).simulate(C())
    got = res.statevector
    assert np.max(np.abs(got - want)) <= d["atol"], (path.stem, exec_mode)
