"""Adjoint gradients and Pauli observables on the GPU (dq_adjoint,
dq_expval_pauli) against the CPU oracle.

Tolerances: observables 1e-12 absolute (FP64, different summation order);
adjoint vs parameter shift 1e-10 (both exact in exact arithmetic); adjoint vs
central finite differences with h = 1e-6: 1e-7 (truncation ~h^2, rounding
~1e-16/h).
"""
import ctypes

import numpy as np
import pytest

import _circuits
import _oracle as orc
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.adjoint import (
    Param,
    ParamCircuit,
    PauliSum,
    adjoint_gradient,
    expectation,
    expval,
    parameter_shift_gradient,
)
from test_adjoint_host import every_kind_circuit

pytestmark = pytest.mark.gpu

TOL_SHIFT = 1e-10
TOL_FD = 1e-7


def random_observable(n, nterms, seed):
    rng = np.random.default_rng(seed)
    H = PauliSum()
    for _ in range(nterms):
        k = int(rng.integers(1, min(n, 4) + 1))
        qs = rng.permutation(n)[:k]
        H.add(float(rng.normal()), {int(q): "XYZ"[rng.integers(3)] for q in qs})
    return H


@pytest.mark.parametrize("n", [3, 11, 14])
def test_expval_pauli_matches_oracle(gpu, n):
    rng = np.random.default_rng(n)
    psi = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    psi /= np.linalg.norm(psi)
    H = random_observable(n, 40, seed=n + 1)
    H.add(0.3, "I")
    st = nat.State(n, 0)
    st.upload(psi)
    out = ctypes.c_double()
    terms = H.array()
    nat.check(nat.lib().dq_expval_pauli(st.handle, nat.ptr(terms), len(terms), ctypes.byref(out)))
    assert abs(out.value - orc.expval_pauli(psi, terms)) < 1e-12


@pytest.mark.parametrize("n,exec_mode", [(3, "per_gate"), (11, "fused"), (11, "per_gate")])
def test_adjoint_every_kind_matches_oracle(gpu, n, exec_mode):
    c, theta = every_kind_circuit(n)
    H = random_observable(n, 10, seed=7)
    e, g = adjoint_gradient(c, theta, H, exec=exec_mode)
    terms = H.array()
    assert abs(e - orc.expval_program(c.bind(theta), n, terms)) < 1e-12
    ps = orc.param_shift(c, theta, terms)
    assert np.max(np.abs(g - ps)) < TOL_SHIFT, np.abs(g - ps)
    fd = orc.finite_difference(c, theta, terms)
    assert np.max(np.abs(g - fd)) < TOL_FD


def test_adjoint_matches_gpu_parameter_shift(gpu):
    c, theta, H = _circuits.hea_param_circuit(12, 3, seed=2)
    e, g = adjoint_gradient(c, theta, H)
    ps = parameter_shift_gradient(c, theta, H, exec="per_gate")
    assert np.max(np.abs(g - ps)) < TOL_SHIFT
    assert abs(e - expectation(c, theta, H)) < 1e-12


def test_adjoint_hea14_matches_oracle_parameter_shift(gpu):
    # the 14-qubit shrink of the 24-qubit, 16-layer HEA workload: full
    # 16-layer gradient checked on a seeded subset of parameters
    c, theta, H = _circuits.hea_param_circuit(14, 16, seed=4)
    e, g = adjoint_gradient(c, theta, H)
    terms = H.array()
    assert abs(e - orc.expval_program(c.bind(theta), 14, terms)) < 1e-12
    sub = sorted(np.random.default_rng(0).choice(len(theta), size=24, replace=False).tolist())
    ps = orc.param_shift(c, theta, terms, occurrences=sub)
    assert np.max(np.abs(g[sub] - ps[sub])) < TOL_SHIFT


def test_shared_and_scaled_parameters(gpu):
    c = ParamCircuit(10, num_params=2)
    for q in range(10):
        c.ry(q, Param(0))
        c.rz(q, Param(1, scale=0.5, shift=0.1))
    for q in range(9):
        c.rzz(q, q + 1, Param(0, scale=-1.5))
    H = PauliSum([(1.0, "Z0 Z1"), (0.5, "X4"), (-0.8, "Y9 Z2")])
    theta = np.array([0.37, -1.2])
    e, g = adjoint_gradient(c, theta, H)
    fd = orc.finite_difference(c, theta, H.array())
    assert np.max(np.abs(g - fd)) < TOL_FD
    ps = orc.param_shift(c, theta, H.array())
    assert np.max(np.abs(g - ps)) < TOL_SHIFT


def test_adjoint_restores_initial_state(gpu):
    c, theta, H = _circuits.hea_param_circuit(12, 4, seed=9)
    tm = {}
    adjoint_gradient(c, theta, H, timing=tm)
    assert set(tm) == {"forward_ms", "observable_ms", "backward_ms", "backward_sweeps"}
    assert all(v > 0 for v in tm.values())
    from dqsim_bosonic_b200 import adjoint as adj

    st = adj._state(12, 0)
    v = st.download()
    assert abs(v[0] - 1.0) < 1e-10 and np.max(np.abs(v[1:])) < 1e-10


def test_torch_autograd_function(gpu):
    import torch

    c, theta, H = _circuits.hea_param_circuit(10, 2, seed=5)
    t = torch.tensor(theta, dtype=torch.float64, requires_grad=True)
    e = expval(t, c, H)
    (2.0 * e).backward()
    _, g = adjoint_gradient(c, theta, H)
    assert torch.allclose(t.grad, torch.from_numpy(2.0 * g), atol=1e-12, rtol=0)
    # batched parameter sets
    tb = torch.tensor(np.stack([theta, theta + 0.1, theta - 0.2]), requires_grad=True)
    eb = expval(tb, c, H)
    assert eb.shape == (3,)
    eb.sum().backward()
    for b in range(3):
        eb_b, gb = adjoint_gradient(c, tb.detach()[b].numpy(), H)
        assert abs(eb[b].item() - eb_b) < 1e-12
        assert np.max(np.abs(tb.grad[b].numpy() - gb)) < 1e-12


def test_adjoint_rejects_non_unitary_programs(gpu):
    st = nat.State(4, 0)
    insts = np.zeros(2, dtype=nat.INST_DTYPE)
    insts["cbit"] = -1
    insts[0]["kind"] = nat.KIND["ry"]; insts[0]["nq"] = 1; insts[0]["p"][0] = 0.3
    insts[1]["kind"] = nat.KIND["measure"]; insts[1]["nq"] = 1; insts[1]["cbit"] = 0
    idx = np.full((2, 4), -1, dtype=np.int32)
    idx[0, 0] = 0
    terms = PauliSum([(1.0, "Z0")]).array()
    e = ctypes.c_double()
    g = np.zeros(1)
    rc = nat.lib().dq_adjoint(st.handle, nat.ptr(insts), 2, nat.ptr(idx), 1, nat.ptr(terms), 1,
                              None, ctypes.byref(e), nat.ptr(g), None)
    assert rc == nat.DQ_ERR_UNSUPPORTED
    # a slot on a kind without that parameter
    insts[1]["kind"] = nat.KIND["h"]; insts[1]["cbit"] = -1
    idx[1, 0] = 0
    rc = nat.lib().dq_adjoint(st.handle, nat.ptr(insts), 2, nat.ptr(idx), 1, nat.ptr(terms), 1,
                              None, ctypes.byref(e), nat.ptr(g), None)
    assert rc == nat.DQ_ERR_INVALID_ARG
    # observable outside the register
    idx[1, 0] = -1
    far = PauliSum([(1.0, "Z7")]).array()
    rc = nat.lib().dq_adjoint(st.handle, nat.ptr(insts), 2, nat.ptr(idx), 1, nat.ptr(far), 1,
                              None, ctypes.byref(e), nat.ptr(g), None)
    assert rc == nat.DQ_ERR_INVALID_ARG


def test_batched_adjoint_matches_single_sets_and_drives_adam(gpu):
    import torch

    from dqsim_bosonic_b200.adjoint import adjoint_gradient_batch

    c, _, H = _circuits.hea_param_circuit(11, 2, seed=3)
    B, P = 6, c.num_params
    thetas = np.random.default_rng(8).uniform(-np.pi, np.pi, size=(B, P))
    es, gs = adjoint_gradient_batch(c, thetas, H, workers=3)
    for b in range(B):
        e1, g1 = adjoint_gradient(c, thetas[b], H)
        assert abs(es[b] - e1) < 1e-13
        assert np.max(np.abs(gs[b] - g1)) < 1e-13
    sub = [0, P // 2, P - 1]
    ps = orc.param_shift(c, thetas[2], H.array(), occurrences=sub)
    assert np.max(np.abs(gs[2][sub] - ps[sub])) < TOL_SHIFT
    # Adam on <H> for every set at once through the autograd function
    t = torch.tensor(thetas, requires_grad=True)
    opt = torch.optim.Adam([t], lr=0.01)
    energies = []
    for _ in range(5):
        opt.zero_grad()
        e = expval(t, c, H, workers=3)
        e.sum().backward()
        opt.step()
        energies.append(e.detach().clone())
    assert energies[-1].sum() < energies[0].sum()


@pytest.mark.parametrize("n,layers,B", [(11, 2, 6), (14, 3, 9), (20, 1, 3)])
def test_batched_launches_match_single_sets(gpu, n, layers, B):
    """dq_adjoint_batch: every sweep index of every set in one launch; energies
    and gradients equal the single-set adjoint pass within 1e-11."""
    from dqsim_bosonic_b200.adjoint import adjoint_gradient_batch

    c, _, H = _circuits.hea_param_circuit(n, layers, seed=3)
    thetas = np.random.default_rng(n).uniform(-np.pi, np.pi, size=(B, c.num_params))
    st = {}
    es, gs = adjoint_gradient_batch(c, thetas, H, stats=st)
    assert st["batched"] == 1 and st["groups"] == 1
    # one launch per forward sweep, one for lambda = H psi, two per backward
    # sweep (the sweep and its gradient reduction), independent of B
    assert st["launches"] == st["forward_sweeps"] + 1 + 2 * st["backward_sweeps"]
    for b in range(B):
        e1, g1 = adjoint_gradient(c, thetas[b], H)
        assert abs(es[b] - e1) < 1e-11
        assert np.max(np.abs(gs[b] - g1)) < 1e-11


def test_batched_shared_scaled_params_and_fallback(gpu):
    from dqsim_bosonic_b200.adjoint import adjoint_gradient_batch

    # shared and scaled parameters, a controlled rotation and a dense two-qubit gate
    n = 12
    c = ParamCircuit(n)
    for q in range(n):
        c.add("ry", [q], [Param(q % 5, scale=0.5, shift=0.1)])
    c.add("crx", [0, 7], [Param(5)])
    c.add("rxx", [3, 11], [Param(6, scale=-2.0)])
    c.add("u3", [9], [Param(7), Param(8), 0.3])
    c.add("rzz", [2, 10], [Param(0)])
    H = random_observable(n, 6, 4)
    thetas = np.random.default_rng(1).uniform(-np.pi, np.pi, size=(4, c.num_params))
    st = {}
    es, gs = adjoint_gradient_batch(c, thetas, H, stats=st)
    assert st["batched"] == 1
    for b in range(4):
        e1, g1 = adjoint_gradient(c, thetas[b], H)
        assert abs(es[b] - e1) < 1e-11 and np.max(np.abs(gs[b] - g1)) < 1e-11
    # fewer than 10 qubits: the set-by-set path, same results
    c2, _, H2 = _circuits.hea_param_circuit(6, 2, seed=2)
    th2 = np.random.default_rng(2).uniform(-np.pi, np.pi, size=(3, c2.num_params))
    st2 = {}
    es2, gs2 = adjoint_gradient_batch(c2, th2, H2, stats=st2)
    assert st2["batched"] == 0
    for b in range(3):
        e1, g1 = adjoint_gradient(c2, th2[b], H2)
        assert abs(es2[b] - e1) < 1e-12 and np.max(np.abs(gs2[b] - g1)) < 1e-12


def mixed_param_circuit(n, depth, seed):
    """Random gates of every kind the ParamCircuit takes (three- to
    five-qubit gates included), every angle of the parametrised ones
    trainable."""
    from dqsim_bosonic_b200.adjoint import _PARAM_COUNT, _QUBITS

    rng = np.random.default_rng(seed)
    kinds = [k for k, q in _QUBITS.items() if q <= n]
    c = ParamCircuit(n)
    k = 0
    for _ in range(depth):
        kind = kinds[rng.integers(len(kinds))]
        qs = [int(v) for v in rng.permutation(n)[:_QUBITS[kind]]]
        npar = _PARAM_COUNT.get(kind, 0)
        c.add(kind, qs, [Param(k + j) for j in range(npar)])
        k += npar
    theta = rng.uniform(-np.pi, np.pi, size=k)
    return c, theta


@pytest.mark.parametrize("n,seed", [(13, 1), (16, 2), (7, 3)])
def test_fused_backward_matches_per_gate_backward(gpu, n, seed):
    c, theta = mixed_param_circuit(n, 160, seed)
    H = random_observable(n, 12, seed=seed + 10)
    e1, g1 = adjoint_gradient(c, theta, H, exec="fused")
    e2, g2 = adjoint_gradient(c, theta, H, exec="per_gate")
    assert abs(e1 - e2) < 1e-12
    assert np.max(np.abs(g1 - g2)) < 1e-11, np.max(np.abs(g1 - g2))
    sub = list(range(0, theta.size, max(1, theta.size // 12)))
    ps = orc.param_shift(c, theta, H.array(), occurrences=sub)
    assert np.max(np.abs(g1[sub] - ps[sub])) < TOL_SHIFT
    from dqsim_bosonic_b200 import adjoint as adj

    v = adj._state(n, 0).download()
    assert abs(v[0] - 1.0) < 1e-10 and np.max(np.abs(v[1:])) < 1e-10


@pytest.mark.parametrize("angle", [0.0, np.pi, -np.pi / 2])
def test_special_angles_keep_their_derivatives(gpu, angle):
    # at these angles some gates are diagonal or the identity while their
    # derivatives are not: the fused planner must not treat them as diagonal
    c, theta = every_kind_circuit(12)
    theta = np.full_like(theta, angle)
    H = random_observable(12, 10, seed=4)
    e1, g1 = adjoint_gradient(c, theta, H, exec="fused")
    e2, g2 = adjoint_gradient(c, theta, H, exec="per_gate")
    assert abs(e1 - e2) < 1e-12
    ps = orc.param_shift(c, theta, H.array())
    assert np.max(np.abs(g1 - ps)) < TOL_SHIFT
    assert np.max(np.abs(g2 - ps)) < TOL_SHIFT


def diagonal_run_circuit(n, depth, seed):
    """Layers of ry then long runs of diagonal gates (trainable and fixed) on
    random qubits: low, middle and high bits, so a run mixes register, lane,
    warp and non-local qubits and runs of more than 64 ops get split."""
    rng = np.random.default_rng(seed)
    c = ParamCircuit(n)
    k = 0
    diag1 = ["rz", "p", "u1", "z", "s", "t", "sdg"]
    diag2 = ["rzz", "cp", "crz", "cu1", "cz"]
    for layer in range(depth):
        for q in range(n):
            c.ry(q, Param(k)); k += 1
        for _ in range(20 + 40 * layer):
            if rng.random() < 0.5:
                kind = diag1[rng.integers(len(diag1))]
                qs = [int(rng.integers(n))]
            else:
                kind = diag2[rng.integers(len(diag2))]
                qs = [int(v) for v in rng.permutation(n)[:2]]
            npar = _PARAM_COUNT_T.get(kind, 0)
            c.add(kind, qs, [Param(k + j) for j in range(npar)])
            k += npar
    theta = rng.uniform(-np.pi, np.pi, size=k)
    return c, theta


_PARAM_COUNT_T = {"rz": 1, "p": 1, "u1": 1, "rzz": 1, "cp": 1, "crz": 1, "cu1": 1}


@pytest.mark.parametrize("n,seed", [(14, 5), (17, 6), (9, 7)])
def test_long_diagonal_runs_match_per_gate_and_parameter_shift(gpu, n, seed):
    c, theta = diagonal_run_circuit(n, 3, seed)
    H = random_observable(n, 12, seed=seed + 20)
    e1, g1 = adjoint_gradient(c, theta, H, exec="fused")
    e2, g2 = adjoint_gradient(c, theta, H, exec="per_gate")
    assert abs(e1 - e2) < 1e-12
    assert np.max(np.abs(g1 - g2)) < 1e-11, np.max(np.abs(g1 - g2))
    sub = list(range(0, theta.size, max(1, theta.size // 16)))
    ps = orc.param_shift(c, theta, H.array(), occurrences=sub)
    assert np.max(np.abs(g1[sub] - ps[sub])) < TOL_SHIFT


def test_diagonal_gates_with_two_trainable_angles(gpu):
    # u3(0, phi, lambda) and cu3(0, phi, lambda) are diagonal with two
    # diagonal derivatives each: both must reach the gradient
    n = 12
    c = ParamCircuit(n)
    k = 0
    for q in range(n):
        c.ry(q, Param(k)); k += 1
    for q in range(n):
        c.add("u3", [q], [0.0, Param(k), Param(k + 1)]); k += 2
    for q in range(n - 1):
        c.add("cu3", [q, q + 1], [0.0, Param(k), Param(k + 1)]); k += 2
        c.add("cu", [q + 1, q], [0.0, Param(k), Param(k + 1), Param(k + 2)]); k += 3
    for q in range(n):
        c.rx(q, Param(k)); k += 1
    theta = np.random.default_rng(3).uniform(-np.pi, np.pi, size=k)
    H = random_observable(n, 10, seed=8)
    e1, g1 = adjoint_gradient(c, theta, H, exec="fused")
    e2, g2 = adjoint_gradient(c, theta, H, exec="per_gate")
    assert abs(e1 - e2) < 1e-12
    assert np.max(np.abs(g1 - g2)) < 1e-11
    ps = orc.param_shift(c, theta, H.array())
    assert np.max(np.abs(g1 - ps)) < TOL_SHIFT


@pytest.mark.parametrize("n,seed", [(11, 1), (13, 2), (17, 3)])
def test_straight_line_phases_match_per_gate(gpu, n, seed):
    # layers of ry and rx on every qubit in a random order, separated by rzz rings: the
    # backward sweeps' register phases of two or three commuting one-parameter ops (real
    # and rx-shaped matrices, every two-op placement of the phase bits), which the fused
    # backward sorts by target and runs as straight-line code
    rng = np.random.default_rng(seed)
    c = ParamCircuit(n)
    k = 0
    for layer in range(4):
        for q in rng.permutation(n):
            (c.rx if layer % 2 else c.ry)(int(q), Param(k))
            k += 1
        for q in range(n):
            c.add("rzz", [q, (q + 1) % n], [Param(k)])
            k += 1
    theta = rng.uniform(-np.pi, np.pi, size=k)
    H = random_observable(n, 10, seed=seed + 20)
    e1, g1 = adjoint_gradient(c, theta, H, exec="fused")
    e2, g2 = adjoint_gradient(c, theta, H, exec="per_gate")
    assert abs(e1 - e2) < 1e-12
    assert np.max(np.abs(g1 - g2)) < 1e-11, np.max(np.abs(g1 - g2))
