"""The MPS oracle (oracle/mps.py) against the reference's MPS test cases and
the statevector oracle (CPU only).

The reference's tests (tests/test_mps_simulation.py, test_mps_converges.py of
the dqsim package) compare the MPS backend with the statevector backend at
1e-8; here the MPS oracle is held to the C statevector oracle at 1e-12 on the
same circuits and on random ones, and the truncation rule is checked on a
hand-computed case.
"""
import math

import numpy as np
import pytest

import _oracle
from _circuits import JsonCircuit, brickwork_u3_cx, cond, g, gate
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

SEED = 42


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


CASES = {
    "product": JsonCircuit(3, [g("h", 0), g("ry", 1, math.pi / 3), g("ry", 2, math.pi / 5)]),
    "non_adjacent_reversed": JsonCircuit(4, [g("h", 0), g("h", 3), g("cx", 3, 1), g("cz", 2, 0),
                                             g("swap", 3, 0), g("cx", 0, 2)]),
    "entangled": JsonCircuit(3, [g("h", 0), g("h", 2), g("ry", 0, 0.123), g("cx", 2, 1), g("cx", 1, 0),
                                 g("swap", 1, 0), g("ry", 2, 0.456), g("cx", 2, 1), g("swap", 2, 1),
                                 g("ry", 1, 0.789), g("cz", 1, 0), g("cx", 0, 1)]),
    "generic_two_qubit": JsonCircuit(4, [g("h", 0), gate("remote_link_psi_minus", [0, 3]),
                                         gate("nonlocal_cz", [3, 1]), gate("remote_cx", [1, 2]),
                                         gate("remote_epr", [2, 0]), gate("remote_barrier", [0, 1])]),
    "brickwork": brickwork_u3_cx(8, 6, seed=3),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_statevector_oracle(name):
    p = prog_of(CASES[name])
    sv, _, dims, _ = _oracle.mps_run(p, SEED)
    ref = _oracle.run(p, SEED)[0]
    assert np.max(np.abs(sv - ref)) < 1e-12
    assert dims[0] == dims[-1] == 1


def test_measurement_and_conditional_pin():
    c = JsonCircuit(2, [g("x", 0), g("measure", 0, 0), cond(0, 1, 1, g("x", 1))], ncbits=1)
    sv, cb, _, _ = _oracle.mps_run(prog_of(c), SEED)
    assert cb.tolist() == [1]
    assert np.allclose(np.abs(sv) ** 2, [0, 0, 0, 1], atol=0)


def test_reset_pin():
    sv, _, _, _ = _oracle.mps_run(prog_of(JsonCircuit(1, [g("x", 0), g("reset", 0)])), SEED)
    assert np.abs(sv[0]) ** 2 == 1.0 and sv[1] == 0


def test_truncation_to_bond_one_keeps_the_dominant_product_state():
    # cos(t) |00> + sin(t) |11> with cos(t) > sin(t): bond 1 keeps |00>, rescaled to norm 1
    t = 0.4
    c = JsonCircuit(2, [g("ry", 0, 2 * t), g("cx", 0, 1)])
    sv, _, dims, _ = _oracle.mps_run(prog_of(c), SEED, max_bond=1)
    assert dims == [1, 1, 1]
    assert abs(abs(sv[0]) - 1.0) < 1e-15 and np.max(np.abs(sv[1:])) < 1e-15


def test_threshold_drops_small_singular_values():
    # singular values cos(t), sin(t) = 1e-7: a threshold above 1e-7 truncates to bond 1
    t = 1e-7
    c = JsonCircuit(2, [g("ry", 0, 2 * t), g("cx", 0, 1)])
    _, _, d_keep, _ = _oracle.mps_run(prog_of(c), SEED, threshold=1e-12)
    _, _, d_drop, _ = _oracle.mps_run(prog_of(c), SEED, threshold=1e-6)
    assert d_keep == [1, 2, 1] and d_drop == [1, 1, 1]


def test_unsupported_instruction_is_reported_with_its_index():
    mod = _oracle.mps_module()
    p = prog_of(JsonCircuit(3, [g("h", 0), g("ccx", 0, 1, 2)]))
    with pytest.raises(mod.Unsupported) as e:
        _oracle.mps_run(p, SEED)
    assert e.value.index == 1


def test_reverse_2q_order_swaps_the_qubit_roles():
    mod = _oracle.mps_module()
    cx = np.eye(4, dtype=complex)[[0, 1, 3, 2]]     # control = first (MSB) qubit
    xc = mod.reverse_2q_order(cx)
    assert np.array_equal(xc, np.eye(4, dtype=complex)[[0, 3, 2, 1]])
