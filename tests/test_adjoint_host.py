"""Host-side pieces of the adjoint-gradient path (no GPU needed).

Pins the checker used by the GPU adjoint tests: the oracle's observable
against dense numpy matrices, and the oracle's parameter-shift gradients
against its own central finite differences for every differentiable kind.
"""
import itertools

import numpy as np
import pytest

import _circuits
import _oracle as orc
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.adjoint import DIFFERENTIABLE_KINDS, Param, ParamCircuit, PauliSum

PAULI = {
    "I": np.eye(2, dtype=complex),
    "X": np.array([[0, 1], [1, 0]], dtype=complex),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "Z": np.array([[1, 0], [0, -1]], dtype=complex),
}


def dense_pauli(n, ops):
    """Kronecker product with qubit 0 as the least significant index bit."""
    m = np.eye(1, dtype=complex)
    for q in reversed(range(n)):
        m = np.kron(m, PAULI[ops.get(q, "I")])
    return m


def test_pauli_sum_masks():
    H = PauliSum([(0.5, "Z0 Z1"), (-1.25, "X3"), (2.0, {2: "Y", 0: "X"}), (0.1, "I"), (0.2, "")])
    a = H.array()
    assert a.dtype == nat.PAULI_DTYPE
    assert list(a["coeff"]) == [0.5, -1.25, 2.0, 0.1, 0.2]
    assert list(a["xmask"]) == [0, 8, 5, 0, 0]
    assert list(a["zmask"]) == [3, 0, 4, 0, 0]
    assert H.num_qubits == 4


@pytest.mark.parametrize("spec", ["Q0", "X", "Z0 Z0", "X-1", "X64"])
def test_pauli_sum_rejects_bad_specs(spec):
    with pytest.raises(ValueError):
        PauliSum([(1.0, spec)])


def test_pauli_sum_rejects_nonfinite():
    with pytest.raises(ValueError):
        PauliSum([(float("nan"), "Z0")])


def test_oracle_expval_matches_dense_matrices():
    rng = np.random.default_rng(3)
    n = 4
    psi = rng.normal(size=16) + 1j * rng.normal(size=16)
    psi /= np.linalg.norm(psi)
    terms = []
    for _ in range(12):
        ops = {q: "IXYZ"[rng.integers(4)] for q in range(n)}
        terms.append((float(rng.normal()), ops))
    H = PauliSum(terms)
    dense = sum(c * dense_pauli(n, ops) for c, ops in terms)
    want = float(np.real(np.vdot(psi, dense @ psi)))
    got = orc.expval_pauli(psi, H.array())
    assert abs(got - want) < 1e-13


def test_param_circuit_bind_and_slots():
    c = ParamCircuit(3)
    c.ry(0, Param(1)).cx(0, 1).u3(2, Param(0), 0.25, Param(1, scale=-2.0, shift=0.5)).rzz(1, 2, 0.7)
    assert c.num_params == 2
    insts = c.bind([0.1, 0.2])
    assert insts.dtype == nat.INST_DTYPE
    assert [nat.KIND_NAMES[k] for k in insts["kind"]] == ["ry", "cx", "u3", "rzz"]
    assert insts[0]["p"][0] == 0.2
    assert list(insts[2]["p"][:3]) == [0.1, 0.25, -2.0 * 0.2 + 0.5]
    assert list(insts[1]["q"][:2]) == [0, 1]
    slots = c.param_slots()
    assert slots.shape == (4, 4)
    assert slots[0, 0] == 0 and slots[2, 0] == 1 and slots[2, 2] == 2
    assert (slots[1] == -1).all() and (slots[3] == -1).all() and slots[2, 1] == -1
    assert [(i, j) for i, j, _ in c.occurrences()] == [(0, 0), (2, 0), (2, 2)]


@pytest.mark.parametrize("bad", [
    lambda c: c.add("ry", [0], []),
    lambda c: c.add("cx", [0, 0]),
    lambda c: c.add("ry", [5], [0.1]),
    lambda c: c.add("measure", [0]),
    lambda c: c.add("rx", [0], [float("inf")]),
    lambda c: c.add("rx", [0], [Param(-1)]),
])
def test_param_circuit_rejects(bad):
    with pytest.raises(ValueError):
        bad(ParamCircuit(3))


def test_bind_checks_theta_length():
    c = ParamCircuit(2).rx(0, Param(0))
    with pytest.raises(ValueError):
        c.bind([0.1, 0.2])


def every_kind_circuit(n=3):
    """One gate of every differentiable kind, each angle trainable, plus
    fixed gates between them."""
    rng = np.random.default_rng(17)
    c = ParamCircuit(n)
    k = 0
    for kind, np_ in DIFFERENTIABLE_KINDS.items():
        nq = 2 if kind in ("crx", "cry", "crz", "cp", "cu1", "cu3", "cu", "rxx", "rzz") else 1
        qs = list(rng.permutation(n)[:nq])
        c.add(kind, qs, [Param(k + j) for j in range(np_)])
        k += np_
        c.h(int(rng.integers(n)))
        c.cx(*[int(v) for v in rng.permutation(n)[:2]])
    theta = rng.uniform(-np.pi, np.pi, size=k)
    return c, theta


def test_oracle_shift_rules_match_finite_differences():
    c, theta = every_kind_circuit()
    H = PauliSum([(0.7, "Z0 Z1"), (-0.4, "X2"), (0.3, "Y1"), (1.1, "X0 Y2")])
    ps = orc.param_shift(c, theta, H.array())
    fd = orc.finite_difference(c, theta, H.array())
    assert np.max(np.abs(ps - fd)) < 1e-8, np.abs(ps - fd)


def test_hea_builder_matches_spec():
    c, theta, H = _circuits.hea_param_circuit(6, 2, seed=1)
    assert c.num_params == 2 * 3 * 6 == theta.size
    kinds = [op[0] for op in c.ops]
    assert kinds[:6] == ["ry"] * 6 and kinds[6:12] == ["rz"] * 6 and kinds[12:18] == ["rzz"] * 6
    assert c.ops[17][1] == (5, 0)
    assert len(H) == 12
    a = H.array()
    assert set(int(x) for x in a["xmask"][6:]) == {1 << q for q in range(6)}
    assert all(int(z) == 0 for z in a["zmask"][6:])
