"""The oracle against known answers (CPU).

The reference's own tests pin the statevector path only through analytic
outcomes of small circuits (tests/test_distribution_e2e.py:167-216,
tests/test_pblock_conditional.py:22-89, tests/test_qasmbench_simulation.py:
91-143, tolerance 1e-6).  Those circuits, their analytic distributions and
the committed golden fixtures are checked here, together with algebraic
properties (unitarity round trips, norm, reset semantics).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

import _oracle
from _circuits import JsonCircuit, cond, g, gate, random_circuit
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

GOLDEN = Path(__file__).resolve().parent / "golden"


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


def probs_of(c, seed=42):
    st, cb, rc, _ = _oracle.run(prog_of(c), seed)
    assert rc == 0
    return np.abs(st) ** 2, cb


def test_bell_pair():
    p, _ = probs_of(JsonCircuit(2, [g("h", 0), g("cx", 0, 1)]))
    assert p[0] == pytest.approx(0.5, abs=1e-12) and p[3] == pytest.approx(0.5, abs=1e-12)
    assert p[1] == 0 and p[2] == 0


def test_x_cx_deterministic():
    p, _ = probs_of(JsonCircuit(2, [g("x", 0), g("cx", 0, 1)]))
    assert p[3] == 1.0


def test_ghz4():
    p, _ = probs_of(JsonCircuit(4, [g("h", 0), g("cx", 0, 1), g("cx", 1, 2), g("cx", 2, 3)]))
    assert p[0] == pytest.approx(0.5, abs=1e-12) and p[15] == pytest.approx(0.5, abs=1e-12)


def test_ry_cx():
    p, _ = probs_of(JsonCircuit(2, [g("ry", 0, math.pi / 3), g("cx", 0, 1)]))
    assert p[0] == pytest.approx(math.cos(math.pi / 6) ** 2, abs=1e-12)
    assert p[3] == pytest.approx(math.sin(math.pi / 6) ** 2, abs=1e-12)


def test_rx_ry_cx():
    p, _ = probs_of(JsonCircuit(2, [g("rx", 0, math.pi / 3), g("ry", 1, math.pi / 4),
                                    g("cx", 0, 1)]))
    a0, a1 = math.cos(math.pi / 6) ** 2, math.sin(math.pi / 6) ** 2
    b0, b1 = math.cos(math.pi / 8) ** 2, math.sin(math.pi / 8) ** 2
    # after cx(0 -> 1): index = q1 q0; q0 = 1 flips q1
    want = np.array([a0 * b0, a1 * b1, a0 * b1, a1 * b0])
    assert np.allclose(p, want, atol=1e-12)


def test_cz_pair_and_xyz():
    p, _ = probs_of(JsonCircuit(2, [g("h", 0), g("h", 1), g("cz", 0, 1)]))
    assert np.allclose(p, 0.25, atol=1e-12)
    st, _, _, _ = _oracle.run(prog_of(JsonCircuit(2, [g("x", 0), g("y", 1), g("z", 0)])), 1)
    # Z X |0> on q0 = -|1>; Y on q1 = i|1>: amplitude of |11> = -i
    assert st[3] == pytest.approx(-1j, abs=1e-15)


def test_conditional_cx_distribution():
    # tests/test_pblock_conditional.py:22-37: measured-control cx gives 00 / 11
    c = JsonCircuit(2, [g("h", 0), g("measure", 0, 0), cond(0, 1, 1, g("cx", 0, 1)),
                        g("measure", 1, 1)], ncbits=2)
    prog = prog_of(c)
    seen = set()
    for seed in range(64):
        _, cb, rc, _ = _oracle.run(prog, seed)
        assert rc == 0
        seen.add((int(cb[0]), int(cb[1])))
    assert seen == {(0, 0), (1, 1)}


def test_conditional_rzz_parametric():
    # tests/test_pblock_conditional.py:67-89: rzz(pi) conditioned on the measured control
    c = JsonCircuit(2, [g("h", 0), g("measure", 0, 0), g("h", 1),
                        cond(0, 1, 1, g("rzz", 0, 1, math.pi)), g("h", 1), g("measure", 1, 1)],
                    ncbits=2)
    prog = prog_of(c)
    for seed in range(64):
        _, cb, rc, _ = _oracle.run(prog, seed)
        assert rc == 0
        assert cb[1] == cb[0]   # rzz(pi) with q0 = 1 acts as Z on q1 up to phase


def test_reset_returns_to_zero():
    c = JsonCircuit(3, [g("h", 0), g("h", 1), g("cx", 1, 2), g("reset", 0), g("reset", 1),
                        g("reset", 2)])
    prog = prog_of(c)
    for seed in range(16):
        st, _, rc, _ = _oracle.run(prog, seed)
        assert rc == 0
        assert abs(st[0]) == pytest.approx(1.0, abs=1e-12)


@pytest.mark.parametrize("seed", range(6))
def test_norm_preserved_random(seed):
    c = random_circuit(seed, 7, 80)
    st, _, rc, _ = _oracle.run(prog_of(c), 0)
    assert rc == 0
    assert np.sum(np.abs(st) ** 2) == pytest.approx(1.0, abs=1e-12)


def test_inverse_round_trip():
    """U then U^dagger restores |0>: cx/ccx/swap are self-inverse, rotations negate."""
    rng = np.random.default_rng(3)
    fwd, inv = [], []
    for _ in range(40):
        k = rng.integers(5)
        a, b, c3 = rng.choice(6, size=3, replace=False).tolist()
        th = float(rng.uniform(-3, 3))
        if k == 0:
            fwd.append(g("rx", a, th)); inv.append(g("rx", a, -th))
        elif k == 1:
            fwd.append(g("cx", a, b)); inv.append(g("cx", a, b))
        elif k == 2:
            fwd.append(g("crz", a, b, th)); inv.append(g("crz", a, b, -th))
        elif k == 3:
            fwd.append(g("ccx", a, b, c3)); inv.append(g("ccx", a, b, c3))
        else:
            fwd.append(g("rzz", a, b, th)); inv.append(g("rzz", a, b, -th))
    c = JsonCircuit(6, [g("h", q) for q in range(6)] + fwd + inv[::-1] + [g("h", q) for q in range(6)])
    st, _, _, _ = _oracle.run(prog_of(c), 0)
    assert abs(st[0]) == pytest.approx(1.0, abs=1e-12)


def test_unsupported_generic_gate_reports_index():
    c = JsonCircuit(2, [g("h", 0), gate("mystery_gate", [0, 1])])
    _, _, rc, failed = _oracle.run(prog_of(c), 0)
    assert rc == -4 and failed == 1


def test_opaque_circuit_gate_is_noop_only_in_shots():
    c = JsonCircuit(2, [g("h", 0), gate("circuit-123", [0, 1]), g("measure", 0, 0)], ncbits=1)
    prog = prog_of(c)
    _, _, rc, failed = _oracle.run(prog, 0)
    assert rc == -4 and failed == 1
    cb, rc2, _ = _oracle.run_shots(prog, 5, 8)
    assert rc2 == 0 and set(cb[:, 0].tolist()) <= {0, 1}


def test_fuse_flushes_before_touching_instruction():
    c = JsonCircuit(2, [g("h", 0), g("t", 0), g("x", 1), g("cx", 0, 1), g("s", 1), g("id", 0)])
    inst, qub, mats = _oracle.fuse(prog_of(c))
    # h,t fused on q0 and x on q1 flushed (in touched order 0, 1) before cx;
    # s on q1 and id on q0 flushed at the end (id alone is dropped as identity)
    assert inst.tolist() == [-1, -1, 3, -1]
    assert qub.tolist()[:2] == [0, 1] and qub.tolist()[3] == 1
    h = np.array([[1, 1], [1, -1]]) / math.sqrt(2)
    t = np.diag([1, np.exp(1j * math.pi / 4)])
    assert np.allclose(mats[0].reshape(2, 2), t @ h, atol=1e-15)


def test_golden_fixtures():
    files = sorted(f for f in GOLDEN.glob("*.json") if not f.name.startswith("amp_"))
    assert files, "golden fixtures missing"
    for f in files:
        fx = json.loads(f.read_text())
        c = JsonCircuit(fx["num_qubits"], fx["circuit"]["instructions"],
                        qregs=fx["circuit"]["qregs"], cregs=fx["circuit"]["cregs"])
        p, _ = probs_of(c, fx.get("seed", 42))
        want = np.zeros_like(p)
        for k, v in fx["probabilities"].items():
            want[int(k)] = v
        assert np.allclose(p, want, atol=fx["atol"]), f.name
