"""MPS backend on the device against the MPS oracle (oracle/mps.py) (needs a B200).

Bars:
  * statevectors (to_statevector of the final MPS) within 1e-12 of the oracle
    without truncation, within 1e-9 with max_bond_dimension truncation (the
    device SVD is one-sided Jacobi, the oracle's LAPACK: the singular vectors
    differ by a gauge, every observable is gauge-invariant up to rounding);
  * identical classical bits for the same seed (outcomes are draw < p1 with
    the same ChaCha8 stream; p1 agrees to ~1e-15);
  * the reference's own MPS test cases (tests/test_mps_simulation.py,
    tests/test_mps_converges.py of the dqsim package) restated on the
    device, with their tolerance (1e-8) or tighter.
"""
import math

import numpy as np
import pytest

import _oracle
from _circuits import JsonCircuit, brickwork_u3_cx, cond, g, gate, random_gate, trajectory_circuit
from dqsim_bosonic_b200 import MpsSimulator, StatevectorSimulator, simulate_monolithic
from dqsim_bosonic_b200 import simulate_monolithic_shots
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode, format_cbits
from dqsim_bosonic_b200.mps import MpsHandle, run_mps_shots

pytestmark = pytest.mark.gpu

SEED = 42


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


def one_two_qubit_circuit(seed, n, depth, measure_every=0):
    """Random one- and two-qubit gates (any pair, either order) with optional
    mid-circuit measure / conditional / reset."""
    rng = np.random.default_rng(seed)
    kinds1 = ["x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "u3", "u", "u2", "u1", "p",
              "rx", "ry", "rz", "id"]
    kinds2 = ["cx", "cz", "cy", "ch", "swap", "csx", "crx", "cry", "crz", "cu1", "cp", "cu3", "cu",
              "rxx", "rzz"]
    insts = []
    for i in range(depth):
        k = kinds1[rng.integers(len(kinds1))] if rng.random() < 0.5 else kinds2[rng.integers(len(kinds2))]
        insts.append(random_gate(rng, n, k))
        if measure_every and i % measure_every == measure_every - 1:
            q = int(rng.integers(n))
            cb = (i // measure_every) % 3
            insts.append(g("measure", q, cb))
            insts.append(cond(cb, 1, 1, g("x", int((q + 1) % n))))
            if rng.random() < 0.5:
                insts.append(g("reset", int(rng.integers(n))))
    return JsonCircuit(n, insts, ncbits=3 if measure_every else 0)


def device_run(c, seed, max_bond=None, thr=1e-12):
    prog = prog_of(c)
    h = MpsHandle(prog.num_qubits, 0, max_bond, thr)
    cbits, st = h.run(prog, seed)
    dims = h.bond_dims()
    sv = h.to_state().download()
    h.release()
    return sv, cbits, dims, st


# ---- the reference's MPS test cases -------------------------------------------------


def _assert_probs_close(a, b, tol=1e-8):
    for s in set(a) | set(b):
        assert abs(a.get(s, 0.0) - b.get(s, 0.0)) < tol


def _assert_mps_matches_statevector(c):
    sv = simulate_monolithic(c, mode="state_vector", seed=SEED)
    mp = simulate_monolithic(c, mode="mps", seed=SEED)
    _assert_probs_close(sv.probabilities(), mp.probabilities())
    assert np.max(np.abs(sv.statevector - mp.statevector)) < 1e-12
    assert abs(sum(mp.probabilities().values()) - 1.0) < 1e-12


def test_product_state():
    _assert_mps_matches_statevector(JsonCircuit(3, [g("h", 0), g("ry", 1, math.pi / 3),
                                                    g("ry", 2, math.pi / 5)]))


def test_non_adjacent_and_reversed_two_qubit_gates():
    _assert_mps_matches_statevector(JsonCircuit(4, [
        g("h", 0), g("h", 3), g("cx", 3, 1), g("cz", 2, 0), g("swap", 3, 0), g("cx", 0, 2)]))


def test_entangled_gates():
    _assert_mps_matches_statevector(JsonCircuit(3, [
        g("h", 0), g("h", 2), g("ry", 0, 0.123), g("cx", 2, 1), g("cx", 1, 0), g("swap", 1, 0),
        g("ry", 2, 0.456), g("cx", 2, 1), g("swap", 2, 1), g("ry", 1, 0.789), g("cz", 1, 0),
        g("cx", 0, 1)]))


def test_mid_circuit_measurement_and_conditional():
    c = JsonCircuit(2, [g("x", 0), g("measure", 0, 0), cond(0, 1, 1, g("x", 1))], ncbits=1)
    r = simulate_monolithic(c, mode="mps", seed=SEED)
    assert r.classical_bits == {0: 1}
    assert r.probabilities() == {3: 1.0}


def test_reset():
    c = JsonCircuit(1, [g("x", 0), g("reset", 0)])
    assert simulate_monolithic(c, mode="mps", seed=SEED).probabilities() == {0: 1.0}


def test_truncated_mps_remains_normalized():
    c = JsonCircuit(4, [g("h", 0), g("h", 1), g("h", 2), g("cx", 0, 3), g("cx", 1, 2),
                        g("ry", 3, 0.77), g("cx", 3, 1)])
    probs = MpsSimulator(seed=SEED, max_bond_dimension=1).simulate(c).probabilities()
    assert all(p >= -1e-12 for p in probs.values())
    assert abs(sum(probs.values()) - 1.0) < 1e-8
    sv, _, dims, _ = device_run(c, SEED, max_bond=1)
    ref, _, rdims, _ = _oracle.mps_run(prog_of(c), SEED, max_bond=1)
    assert dims == rdims == [1] * 5
    assert np.max(np.abs(sv - ref)) < 1e-9


def test_convenience_function_accepts_mps_bond_dimension():
    c = JsonCircuit(3, [g("h", 0), g("h", 1), g("cx", 0, 2), g("cx", 1, 2)])
    probs = simulate_monolithic(c, mode="mps", seed=SEED, max_bond_dimension=1,
                                truncation_threshold=1e-12).probabilities()
    assert all(p >= -1e-12 for p in probs.values())
    assert abs(sum(probs.values()) - 1.0) < 1e-8


def test_unsupported_multi_qubit_gate_raises():
    c = JsonCircuit(3, [g("h", 0), g("ccx", 0, 1, 2)])
    with pytest.raises(NotImplementedError, match="one- and two-qubit"):
        simulate_monolithic(c, mode="mps", seed=SEED)


def test_unsupported_generic_gate_raises_with_its_name():
    c = JsonCircuit(2, [g("h", 0), gate("Weird_Gate", [0, 1])])
    with pytest.raises(NotImplementedError, match='does not support generic gate "weird_gate"'):
        simulate_monolithic(c, mode="mps", seed=SEED)
    with pytest.raises(NotImplementedError, match="generic gate"):
        simulate_monolithic_shots(c, mode="mps", shots=4, seed=SEED)


def test_unsupported_gate_only_raises_when_its_condition_holds():
    never = JsonCircuit(3, [g("measure", 0, 0), cond(0, 1, 1, g("ccx", 0, 1, 2)), g("h", 1)], ncbits=1)
    r = simulate_monolithic(never, mode="mps", seed=SEED)
    assert r.classical_bits == {0: 0}
    fires = JsonCircuit(3, [g("x", 0), g("measure", 0, 0), cond(0, 1, 1, g("ccx", 0, 1, 2))], ncbits=1)
    with pytest.raises(NotImplementedError, match="one- and two-qubit"):
        simulate_monolithic(fires, mode="mps", seed=SEED)


def _high_entanglement_circuit():
    insts = [g("h", q) for q in range(6)]
    pairs = [(0, 5), (1, 4), (2, 3), (0, 2), (3, 5), (1, 3)]
    for layer in range(3):
        for c_, t in pairs:
            insts.append(g("cx", c_, t))
        for q in range(6):
            insts.append(g("ry", q, 0.2 * (layer + 1) * (q + 1)))
    return JsonCircuit(6, insts)


def _measured_entanglement_circuit():
    insts = [g("h", q) for q in range(4)]
    pairs = [(0, 3), (1, 2), (0, 2), (3, 1)]
    for layer in range(2):
        for c_, t in pairs:
            insts.append(g("cx", c_, t))
        for q in range(4):
            insts.append(g("ry", q, 0.3 * (layer + 1) * (q + 1)))
    insts += [g("measure", q, q) for q in range(4)]
    return JsonCircuit(4, insts, ncbits=4)


def _l1(a, b):
    return sum(abs(a.get(s, 0.0) - b.get(s, 0.0)) for s in set(a) | set(b))


# The reference's convergence tests also use bond dimension 3.  There one
# truncation of the 6-qubit circuit cuts between two equal singular values
# (0.429008, 0.429008), so which of the two directions survives is a choice of
# the SVD routine (nalgebra's, LAPACK's and the device Jacobi's differ); the
# restated tests use the bond dimensions whose truncations are unique.
CONVERGENCE_BONDS = [2, 4, 8]


def test_full_distribution_converges_as_bond_dimension_increases():
    c = _high_entanglement_circuit()
    exact = simulate_monolithic(c, mode="state_vector", seed=SEED).probabilities()
    errs = [_l1(exact, simulate_monolithic(c, mode="mps", seed=SEED, max_bond_dimension=chi).probabilities())
            for chi in CONVERGENCE_BONDS]
    assert errs[1] < errs[0]
    assert errs[2] < 1e-10


def test_marginals_converge_for_ordered_and_reordered_qubit_lists():
    c = _high_entanglement_circuit()
    sv = simulate_monolithic(c, mode="state_vector", seed=SEED)
    res = {chi: simulate_monolithic(c, mode="mps", seed=SEED, max_bond_dimension=chi)
           for chi in CONVERGENCE_BONDS}
    for qubits in ([1, 3], [3, 1], [5, 2, 0]):
        exact = sv.probabilities(list(qubits))
        errs = [_l1(exact, res[chi].probabilities(list(qubits))) for chi in CONVERGENCE_BONDS]
        assert errs[1] < errs[0]
        assert errs[2] < 1e-10


def test_measurement_shot_distribution_converges_with_bond_dimension():
    c = _measured_entanglement_circuit()
    shots = 300
    sv_counts = simulate_monolithic_shots(c, mode="state_vector", shots=shots, seed=SEED)
    errs = []
    for chi in (1, 2, 4):
        mp = simulate_monolithic_shots(c, mode="mps", shots=shots, seed=SEED, max_bond_dimension=chi)
        assert sum(mp.values()) == shots
        errs.append(_l1(sv_counts, mp) / shots)
    assert errs[1] < errs[0]
    assert errs[2] < 1e-10


# ---- parity with the MPS oracle ------------------------------------------------------


@pytest.mark.parametrize("seed,n,depth", [(1, 5, 60), (2, 8, 120), (3, 10, 160), (4, 12, 200)])
def test_random_circuits_match_oracle(seed, n, depth):
    c = one_two_qubit_circuit(seed, n, depth)
    sv, _, dims, st = device_run(c, SEED)
    ref, _, rdims, calls = _oracle.mps_run(prog_of(c), SEED)
    assert np.max(np.abs(sv - ref)) < 1e-12
    assert dims == rdims
    assert st.svd_calls == calls


@pytest.mark.parametrize("max_bond,thr", [(2, 1e-12), (3, 1e-12), (5, 1e-12), (None, 1e-3)])
def test_truncation_matches_oracle(max_bond, thr):
    c = brickwork_u3_cx(10, 8, seed=11)
    sv, _, dims, _ = device_run(c, SEED, max_bond=max_bond, thr=thr)
    ref, _, rdims, _ = _oracle.mps_run(prog_of(c), SEED, max_bond=max_bond, threshold=thr)
    assert dims == rdims
    # (truncation rescales theta to its full norm, not the state: the norm
    # of the truncated state is not 1, in the reference as here)
    assert np.max(np.abs(sv - ref)) < 1e-9


def test_capacity_growth_to_global_work_area_matches_oracle():
    # bond dimension 64 at the middle of 12 qubits: the handle starts at
    # capacity 16 and re-runs at 32 and 64 (64: SVD work area in global memory)
    c = brickwork_u3_cx(12, 14, seed=3)
    sv, _, dims, st = device_run(c, SEED)
    ref, _, rdims, _ = _oracle.mps_run(prog_of(c), SEED)
    assert max(dims) == 64 and st.capacity == 64
    assert dims == rdims
    assert np.max(np.abs(sv - ref)) < 1e-12


def test_bond_128_matches_oracle():
    # capacity 128: theta up to 256 x 256
    c = brickwork_u3_cx(14, 14, seed=4)
    sv, _, dims, st = device_run(c, SEED)
    ref, _, rdims, _ = _oracle.mps_run(prog_of(c), SEED)
    assert max(dims) == 128 and st.capacity == 128
    assert dims == rdims
    assert np.max(np.abs(sv - ref)) < 1e-12


@pytest.mark.parametrize("seed", [5, 6, 7])
def test_measurements_match_oracle(seed):
    c = one_two_qubit_circuit(seed, 7, 90, measure_every=9)
    prog = prog_of(c)
    for s in (SEED, 1000 + seed):
        sv, cbits, _, _ = device_run(c, s)
        ref, rcb, _, _ = _oracle.mps_run(prog, s)
        assert cbits.tolist() == rcb.tolist()
        assert np.max(np.abs(sv - ref)) < 1e-11


def test_shots_match_oracle_per_shot():
    c = trajectory_circuit(8, 9, seed=5)
    prog = prog_of(c)
    shots = 48
    bits, st = run_mps_shots(prog, 99, shots, 0, None, 1e-12, batch=20)  # 3 launches of <= 20
    for i in range(shots):
        _, rcb, _, _ = _oracle.mps_run(prog, 99 + i)
        assert bits[i].tolist() == rcb.tolist(), i
    counts = MpsSimulator(seed=99).simulate_shots(c, shots)
    ref_counts = {}
    for i in range(shots):
        k = format_cbits(bits[i], prog.num_cbits)
        ref_counts[k] = ref_counts.get(k, 0) + 1
    assert counts == ref_counts


@pytest.mark.parametrize("max_bond", [3, 16, 32])
def test_large_batch_steps_match_oracle(max_bond):
    # 600 replicas per launch: bonds <= 16 take the two-warps-per-replica form of
    # the fused step, bond 32 the 256-thread CTA form
    c = trajectory_circuit(10, 9, seed=8)
    prog = prog_of(c)
    bits, st = run_mps_shots(prog, 5, 600, 0, max_bond, 1e-12)
    assert st.replicas == 600 and st.capacity <= max(16, max_bond)
    for i in list(range(12)) + [299, 300, 599]:
        _, rcb, _, _ = _oracle.mps_run(prog, 5 + i, max_bond=max_bond)
        assert bits[i].tolist() == rcb.tolist(), i


def test_shots_agree_with_statevector_distribution():
    c = JsonCircuit(4, [g("h", q) for q in range(4)] + [g("cx", 0, 3), g("cx", 1, 2), g("ry", 0, 0.6),
                                                      g("cx", 3, 1)] +
                    [g("measure", q, q) for q in range(4)], ncbits=4)
    shots = 4000
    mp = simulate_monolithic_shots(c, mode="mps", shots=shots, seed=3)
    sv = StatevectorSimulator(seed=3).simulate_shots(c, shots)
    l1 = sum(abs(mp.get(k, 0) - sv.get(k, 0)) for k in set(mp) | set(sv)) / shots
    assert l1 < 0.08


def test_apply_2q_primitive_matches_oracle():
    c = brickwork_u3_cx(6, 4, seed=2)
    prog = prog_of(c)
    h = MpsHandle(6, 0, None, 1e-12)
    h.run(prog, SEED)
    rng = np.random.default_rng(0)
    m = rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))
    u, _ = np.linalg.qr(m)
    h.apply_2q(4, 1, u)
    sv = h.to_state().download()
    mod = _oracle.mps_module()
    ref_mps, _ = mod.run(prog.insts, prog.conds, 6, prog.cbit_space, _oracle._Draws(SEED),
                         _oracle._mps_classify)
    ref_mps.apply_2q(4, 1, u, np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]])
    assert np.max(np.abs(sv - ref_mps.to_statevector())) < 1e-12
    assert h.bond_dims() == ref_mps.bond_dims()
    h.release()


def test_shot_slices_reproduce_the_full_run():
    # shot i is seeded base + i whatever the batch or the rank split: rows of a
    # slice run equal the same rows of the full run (the sharded path relies on it)
    from dqsim_bosonic_b200.dist import simulate_shots_sharded

    c = trajectory_circuit(9, 6, seed=2)
    prog = prog_of(c)
    full, _ = run_mps_shots(prog, 41, 400, 0, 8, 1e-12)
    part, _ = run_mps_shots(prog, 41 + 150, 100, 0, 8, 1e-12)
    assert np.array_equal(full[150:250], part)
    sim = MpsSimulator(seed=41, max_bond_dimension=8)
    assert simulate_shots_sharded(sim, c, 400) == sim.simulate_shots(c, 400)


def test_generic_gates_and_nested_conditionals_match_oracle():
    insts = [g("h", 0), g("h", 2), gate("remote_link_psi_minus", [0, 3]), gate("nonlocal_cz", [3, 1]),
             gate("remote_cx", [1, 2]), gate("remote_epr", [2, 0]), gate("remote_barrier", [0, 1]),
             gate("circuit-opaque", [0, 1, 2]), g("ry", 0, 1.1), g("ry", 2, 0.7), g("cx", 0, 2),
             g("measure", 0, 0), g("measure", 2, 1),
             cond(0, 1, 1, cond(1, 1, 0, g("x", 3))), cond(0, 2, 3, gate("remote_cz", [1, 3])),
             g("ry", 1, 0.3), g("measure", 3, 2)]
    c = JsonCircuit(4, insts, ncbits=3)
    prog = prog_of(c)
    for s in range(6):
        sv, cb, dims, _ = device_run(c, s)
        ref, rcb, rdims, _ = _oracle.mps_run(prog, s)
        assert cb.tolist() == rcb.tolist()
        assert dims == rdims
        assert np.max(np.abs(sv - ref)) < 1e-12


def test_shots_beyond_statevector_width_ghz40():
    # 40 qubits (no statevector of that size exists): GHZ by h + a cx chain (bond
    # dimension 2), then every qubit measured; each shot reads all zeros or all ones
    n = 40
    insts = [g("h", 0)] + [g("cx", i, i + 1) for i in range(n - 1)] + [g("measure", i, i) for i in range(n)]
    c = JsonCircuit(n, insts, ncbits=n)
    counts = MpsSimulator(seed=9).simulate_shots(c, 2000)
    assert set(counts) <= {"0" * n, "1" * n}
    assert sum(counts.values()) == 2000
    assert 800 < counts.get("1" * n, 0) < 1200
    # reset + conditional across the chain: flip qubit 39 back when qubit 0 read 1
    insts2 = insts[:n] + [g("measure", 0, 0), cond(0, 1, 1, g("x", n - 1)), g("measure", n - 1, 1)]
    c2 = JsonCircuit(n, insts2, ncbits=2)
    counts2 = MpsSimulator(seed=9).simulate_shots(c2, 500)
    assert set(counts2) <= {"00", "01"}


def test_threshold_extremes_follow_the_keep_rule():
    # negative: every singular value kept (exact state); NaN / +inf: one kept (bond 1)
    c = brickwork_u3_cx(6, 4, seed=6)
    prog = prog_of(c)
    exact = _oracle.run(prog, SEED)[0]
    _, _, edims, _ = _oracle.mps_run(prog, SEED, threshold=-1.0)
    sv, _, dims, _ = device_run(c, SEED, thr=-1.0)
    assert dims == edims == [1, 2, 4, 8, 4, 2, 1]
    assert np.max(np.abs(sv - exact)) < 1e-12
    for thr in (float("nan"), float("inf")):
        sv1, _, d1, _ = device_run(c, SEED, thr=thr)
        ref1, _, r1, _ = _oracle.mps_run(prog, SEED, threshold=thr)
        assert d1 == r1 == [1] * 7
        assert np.max(np.abs(sv1 - ref1)) < 1e-9


def test_apply_2q_widens_a_live_handle():
    # 10 qubits (bond bound 32, starting capacity 16): a brickwork run reaches bond 16,
    # then long-range gates push a bond to 32, so dq_mps_apply_2q widens the live
    # handle (dq_mps_reserve keeps its state) and redoes the overflowing step
    c = brickwork_u3_cx(10, 6, seed=12)
    prog = prog_of(c)
    h = MpsHandle(10, 0, None, 1e-12)
    h.run(prog, SEED)
    mod = _oracle.mps_module()
    ref, _ = mod.run(prog.insts, prog.conds, 10, prog.cbit_space, _oracle._Draws(SEED),
                     _oracle._mps_classify)
    swap = np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    rng = np.random.default_rng(3)
    for a, b in ((0, 9), (8, 1), (2, 7), (6, 3)):
        u, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
        h.apply_2q(a, b, u)
        ref.apply_2q(a, b, u, swap)
    assert max(h.bond_dims()) == 32
    assert h.bond_dims() == ref.bond_dims()
    assert np.max(np.abs(h.to_state().download() - ref.to_statevector())) < 1e-12
    h.release()


@pytest.mark.parametrize("thr", [0.0, -1.0])
def test_rank_deficient_thetas_at_rounding_threshold_match_exact_state(thr):
    # A GHZ chain makes every theta rank 2 and the swap chains of long-range gates
    # move product-like bonds: their other singular values sit at the rounding level,
    # and a threshold of 0 (or below) keeps them.  Such kept columns are written as
    # zeros by the split, so later steps see no O(1) non-isometric entries: the
    # state after further entangling gates still equals the exact statevector.
    n = 8
    rng = np.random.default_rng(11)
    insts = [g("h", 0)] + [g("cx", q, q + 1) for q in range(n - 1)]
    insts += [g("swap", 0, 5), g("swap", 7, 2), g("cx", 1, 6), g("cz", 6, 0)]
    insts += [random_gate(rng, n, "u3") for _ in range(n)]
    insts += [g("rzz", 3, 4, 0.3), g("cx", 0, 7), g("swap", 2, 6)]
    insts += [random_gate(rng, n, "ry") for _ in range(n)]
    c = JsonCircuit(n, insts)
    prog = prog_of(c)
    exact = _oracle.run(prog, SEED)[0]
    sv, _, dims, _ = device_run(c, SEED, thr=thr)
    assert np.max(np.abs(sv - exact)) < 1e-12
    assert abs(np.vdot(sv, sv).real - 1.0) < 1e-12
    assert max(dims) <= 16
