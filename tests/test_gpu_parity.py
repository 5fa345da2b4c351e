"""Parity of the CUDA engine with the CPU oracle (needs a B200).

Bars (the statevector path's contract):
  * per-gate execution: amplitudes bit-identical to the oracle for unitary
    programs (same operation order, no FMA) -- compared with array_equal;
  * programs with measurements: identical outcomes and classical bits, and
    amplitudes within 1e-12 (the p1 sum order of a parallel reduction
    differs from any sequential one, so the collapse divides by a norm that
    can differ in the last bit);
  * sampling: identical indices except draws within 1e-12 of a CDF
    boundary, which the engine counts and reports.
"""
import ctypes
import math

import numpy as np
import pytest

import _oracle
from _circuits import (GATE_ARITY, GATE_NPARAMS, QUBIT_FIELDS, UNITARY_KINDS, JsonCircuit,
                       brickwork_u3_cx, cond, g, gate, random_circuit, random_gate,
                       trajectory_circuit, _FIELDS)
from dqsim_bosonic_b200 import StatevectorSimulator
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
from dqsim_bosonic_b200.statevector import run_program

pytestmark = pytest.mark.gpu

ATOL = 1e-12


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def gpu_run(prog, seed, init=None, exec_mode=nat.EXEC_PER_GATE, semantics=nat.SEM_SIMULATE):
    st = nat.State(prog.num_qubits, 0)
    if init is not None:
        st.upload(init)
    cbits, prof = run_program(st, prog, seed, semantics, exec_mode)
    out = st.download()
    st.release()
    return out, cbits, prof


def all_placements(kind, n, rng, count):
    k = GATE_ARITY[kind]
    out = []
    for _ in range(count):
        qs = rng.choice(n, size=k, replace=False).tolist()
        ps = rng.uniform(-2 * math.pi, 2 * math.pi, size=GATE_NPARAMS[kind]).tolist()
        vals, qi, pi = [], 0, 0
        for f in _FIELDS[kind]:
            if f in QUBIT_FIELDS:
                vals.append(qs[qi]); qi += 1
            else:
                vals.append(ps[pi]); pi += 1
        out.append(g(kind, *vals))
    return out


@pytest.mark.parametrize("kind", [k for k in UNITARY_KINDS])
def test_every_gate_bit_exact(gpu, kind):
    n = 7
    rng = np.random.default_rng(sum(map(ord, kind)))
    insts = all_placements(kind, n, rng, 12)
    init = random_state(n, 11)
    prog = prog_of(JsonCircuit(n, insts))
    want, _, rc, _ = _oracle.run(prog, 0, init)
    assert rc == 0
    got, _, _ = gpu_run(prog, 0, init)
    assert np.array_equal(got, want), f"{kind}: max diff {np.max(np.abs(got - want))}"


@pytest.mark.parametrize("name", ["remote_link_phi_plus", "remote_link_psi_minus",
                                  "remote_link_psi_plus", "nonlocal_cz", "remote_cz",
                                  "remote_cx", "remote_epr", "remote_barrier", "REMOTE_CU1"])
def test_generic_gates_bit_exact(gpu, name):
    n = 6
    init = random_state(n, 5)
    insts = [gate(name, [a, b]) for a, b in ((0, 5), (5, 0), (2, 3), (4, 1))]
    prog = prog_of(JsonCircuit(n, insts))
    want, _, rc, _ = _oracle.run(prog, 0, init)
    assert rc == 0
    got, _, _ = gpu_run(prog, 0, init)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n,depth,seed", [(1, 30, 1), (3, 60, 2), (9, 300, 3), (12, 300, 4),
                                          (14, 200, 5)])
def test_random_circuits_bit_exact(gpu, n, depth, seed):
    prog = prog_of(random_circuit(seed, n, depth))
    want, _, _, _ = _oracle.run(prog, 0)
    got, _, _ = gpu_run(prog, 0)
    assert np.array_equal(got, want)


def test_zero_qubit_circuit(gpu):
    c = JsonCircuit(0, [], qregs={})
    res = StatevectorSimulator(seed=1).simulate(c)
    assert res.num_qubits == 0
    assert res.statevector.tolist() == [1 + 0j]
    assert res.probabilities() == {0: 1.0}
    assert res.counts(shots=5, seed=3) == {"0": 5}


def measured_program(seed, n=8, layers=6):
    rng = np.random.default_rng(seed)
    insts = []
    for layer in range(layers):
        for q in range(n):
            insts.append(g("u3", q, *rng.uniform(0, 2 * math.pi, 3).tolist()))
        for q in range(layer % 2, n - 1, 2):
            insts.append(g("cx", q, q + 1))
        insts.append(g("measure", layer % n, layer % 3))
        insts.append(cond(layer % 3, 1, 1, g("x", (layer + 1) % n)))
        insts.append(cond(0, 2, 2, g("rzz", 0, n - 1, 0.3)))
        if layer % 2:
            insts.append(g("reset", (layer + 2) % n))
    insts.append(g("measure", 1, 4))
    return JsonCircuit(n, insts, ncbits=5)


@pytest.mark.parametrize("seed", range(8))
def test_measure_reset_conditional_match(gpu, seed):
    prog = prog_of(measured_program(seed))
    for rseed in (seed, 1000 + seed):
        want, wcb, rc, _ = _oracle.run(prog, rseed)
        got, gcb, prof = gpu_run(prog, rseed)
        if prof.boundary_draws:
            continue
        assert gcb.tolist() == wcb.tolist()
        assert np.max(np.abs(got - want)) < ATOL


def test_shots_semantics_match_oracle(gpu):
    c = trajectory_circuit(n=8, layers=6, seed=3)
    prog = prog_of(c)
    from dqsim_bosonic_b200.batch import run_trajectories

    bits, _, _ = run_trajectories(prog, 77, 48, 0)
    want, rc, _ = _oracle.run_shots(prog, 77, 48)
    assert rc == 0
    assert bits.tolist() == want.tolist()


@pytest.mark.parametrize("qubits", [None, [0], [3, 1], [5, 0, 2], [7, 6, 5, 4], [2, 7, 0, 5, 1, 3]])
def test_marginal_probabilities(gpu, qubits):
    n = 8
    init = random_state(n, 21)
    st = nat.State(n, 0)
    st.upload(init)
    from dqsim_bosonic_b200.statevector import SimulationResult

    res = SimulationResult(st, n, {}, None)
    qs = list(range(n - 1, -1, -1)) if qubits is None else qubits
    want = _oracle.marginal(init, qs)
    got = res.probability_array(qubits)
    nterms = 1 << (n - len(qs))
    if nterms <= 64:
        assert np.array_equal(got, want)
    else:
        assert np.max(np.abs(got - want)) < ATOL


def test_marginal_large_reduction(gpu):
    n = 20
    init = random_state(n, 2)
    st = nat.State(n, 0)
    st.upload(init)
    from dqsim_bosonic_b200.statevector import SimulationResult

    res = SimulationResult(st, n, {}, None)
    for qs in ([19], [0, 10], [3, 17, 8], list(range(10)), [7, 0, 3], [9, 1]):
        want = _oracle.marginal(init, qs)
        got = res.probability_array(qs)
        assert np.max(np.abs(got - want)) < ATOL
    assert res.probability_array([]).tolist() == pytest.approx([1.0], abs=1e-12)


@pytest.mark.parametrize("qubits,seed", [(None, 7), ([2, 0], 3), ([5, 1, 3], 99)])
def test_sampling_matches_oracle(gpu, qubits, seed):
    n = 10
    init = random_state(n, 4)
    st = nat.State(n, 0)
    st.upload(init)
    from dqsim_bosonic_b200.statevector import SimulationResult

    res = SimulationResult(st, n, {}, None)
    qs = list(range(n - 1, -1, -1)) if qubits is None else qubits
    got = res.sample_indices(4000, qubits, seed)
    want = _oracle.sample(init, qs, seed, 4000)
    mism = int(np.sum(got != want))
    assert mism <= res.last_boundary_draws
    k = len(qs)
    c = res.counts(4000, qubits, seed)
    assert sum(c.values()) == 4000 and all(len(key) == k for key in c)


def test_fidelity_and_norm(gpu):
    n = 9
    a = random_state(n, 1)
    b = random_state(n, 2)
    st = nat.State(n, 0)
    st.upload(a)
    from dqsim_bosonic_b200.statevector import SimulationResult

    res = SimulationResult(st, n, {}, None)
    assert res.fidelity(b) == pytest.approx(abs(np.vdot(a, b)) ** 2, abs=1e-13)
    assert res.fidelity(a) == pytest.approx(1.0, abs=1e-12)
    assert res.fidelity(np.zeros(4, dtype=np.complex128)) == 0.0
    with pytest.raises(TypeError):
        res.fidelity(np.zeros(1 << n, dtype=np.complex64))


def test_apply_1q_with_zero_controls(gpu, engine_lib):
    n = 6
    init = random_state(n, 8)
    u = np.array([0.6, 0.8j, 0.8j, 0.6], dtype=np.complex128)
    want = init.copy()
    _oracle.apply_one_qubit(want, u, 2, incl=(1 << 0) | (1 << 4), desired=(1 << 4))
    st = nat.State(n, 0)
    st.upload(init)
    nat.check(engine_lib.dq_apply_1q(st.handle, u.ctypes.data, 2, (1 << 0) | (1 << 4), 1 << 4))
    assert np.array_equal(st.download(), want)


def test_apply_dense_matches_oracle(gpu, engine_lib):
    n = 7
    rng = np.random.default_rng(0)
    for k in range(1, 6):
        m = rng.normal(size=(1 << k, 1 << k)) + 1j * rng.normal(size=(1 << k, 1 << k))
        m[rng.random(m.shape) < 0.3] = 0
        qs = rng.choice(n, size=k, replace=False).astype(np.uint32)
        init = random_state(n, k)
        want = init.copy()
        _oracle.apply_n_qubit(want, m, qs)
        st = nat.State(n, 0)
        st.upload(init)
        mm = np.ascontiguousarray(m)
        nat.check(engine_lib.dq_apply_dense(st.handle, mm.ctypes.data, qs.ctypes.data, k))
        assert np.array_equal(st.download(), want), k


def test_errors_surface_as_reference_exceptions(gpu):
    sim = StatevectorSimulator(seed=1)
    with pytest.raises(NotImplementedError, match='Unsupported generic gate: "mystery"'):
        sim.simulate(JsonCircuit(2, [g("h", 0), gate("Mystery", [0, 1])]))
    with pytest.raises(RuntimeError, match="Unsupported generic gate"):
        sim.simulate_shots(JsonCircuit(2, [gate("mystery", [0, 1])]), shots=2)
    with pytest.raises(ValueError, match="out of range"):
        sim.simulate(JsonCircuit(2, [g("x", 2)]))
    with pytest.raises(ValueError, match="Circuit JSON parse error"):
        sim.simulate(JsonCircuit(2, [{"kind": "x"}]))
    # a conditional unsupported gate that never fires is not an error
    c = JsonCircuit(2, [cond(0, 1, 1, gate("mystery", [0, 1]))], ncbits=1)
    assert sim.simulate(c).probabilities() == {0: 1.0}


def test_profile_counts_kernel_classes(gpu):
    c = JsonCircuit(3, [g("h", 0), g("cx", 0, 1), g("measure", 1, 0), g("reset", 2), g("rz", 2, 0.1)],
                    ncbits=1)
    res = StatevectorSimulator(seed=3, profile=True).simulate(c)
    p = res.profile
    assert p.apply_n_qubit_calls == 1
    assert p.measure_qubit_calls == 2
    assert p.apply_one_qubit_calls >= 2
    assert p.total_time >= p.apply_one_qubit_time >= 0.0
    assert "SimulationProfile (total:" in repr(p)


def test_brickwork20_full_size_bit_exact(gpu):
    """20-qubit u3+cx brickwork, 20 layers: statevector, probabilities and
    counts(10000, seed=7) against the oracle (per-gate execution)."""
    c = brickwork_u3_cx(20, 20, 1234)
    prog = prog_of(c)
    _oracle.set_threads(8)
    want, _, rc, _ = _oracle.run(prog, 0)
    assert rc == 0
    res = StatevectorSimulator(seed=0, exec="per_gate").simulate(c)
    got = res.statevector
    assert np.array_equal(got, want)
    probs = res.probability_array()
    assert np.array_equal(probs, _oracle.marginal(want, list(range(19, -1, -1))))
    idx = res.sample_indices(10000, None, 7)
    widx = _oracle.sample(want, list(range(19, -1, -1)), 7, 10000)
    assert int(np.sum(idx != widx)) <= res.last_boundary_draws
