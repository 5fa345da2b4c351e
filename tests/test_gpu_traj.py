"""Batched trajectories (dq_run_trajectories, dq_run_batch) against the oracle.

Classical registers must equal the oracle's sequential shots bit for bit,
except for draws within 1e-12 of p1 (reported as boundary draws; the p1 sums
run in different orders).  Final states of unitary batch items match within
1e-12 (shot-semantics fusion vs the simulate path).
"""
import numpy as np
import pytest

import _circuits
import _oracle as orc
from _circuits import JsonCircuit, cond, g
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.batch import (
    TrajectoryPlan,
    TrajectoryTuner,
    _opts,
    run_batch,
    run_trajectories,
    trajectories_resident,
)
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

pytestmark = pytest.mark.gpu


def prog_of(circ):
    return encode(decode_circuit_json(circ.model_dump_json()))


def shot_circuit(n, depth, seed, ncbits=4):
    """Random gates of every kind with measurements, resets and conditionals
    on random qubits (cluster qubits included)."""
    rng = np.random.default_rng(seed)
    insts = []
    for _ in range(depth):
        r = rng.random()
        if r < 0.12:
            insts.append(g("measure", int(rng.integers(n)), int(rng.integers(ncbits))))
        elif r < 0.18:
            insts.append(g("reset", int(rng.integers(n))))
        elif r < 0.28:
            base = int(rng.integers(ncbits - 1))
            insts.append(cond(base, 2, int(rng.integers(4)), _circuits.random_gate(rng, n)))
        else:
            insts.append(_circuits.random_gate(rng, n))
    for q in range(min(n, ncbits)):
        insts.append(g("measure", q, q))
    return JsonCircuit(n, insts, ncbits=ncbits)


def assert_cbits_match(got, want, boundary):
    bad = int(np.sum(np.any(got != want, axis=1)))
    assert bad <= boundary, (bad, boundary)


@pytest.mark.parametrize("n,local_bits,threads", [
    (3, 0, 128), (8, 0, 256), (10, 0, 512), (12, 9, 256), (11, 8, 128),
    (13, 0, 256), (14, 0, 256), (15, 0, 512), (16, 0, 256),
])
def test_trajectories_match_oracle(gpu, n, local_bits, threads):
    prog = prog_of(shot_circuit(n, 60, seed=100 + n))
    shots = 48
    want, rc, _ = orc.run_shots(prog, 7, shots)
    assert rc == 0
    got, st = trajectories_resident(prog, 7, shots, opts=_opts(threads, 8, local_bits))
    assert st.cluster_span == 1 << (n - (local_bits or min(n, 13)))
    assert_cbits_match(got, want, st.boundary_draws)


def test_trajectory_workload_16q_matches_oracle(gpu):
    # 12 layers of u3 + cx brickwork, measure q0 / conditional x q1 / reset q0
    # after every third layer: the 16-qubit batched-trajectory workload
    prog = prog_of(_circuits.trajectory_circuit(16, 12, seed=7))
    shots = 256
    want, rc, _ = orc.run_shots(prog, 7, shots)
    assert rc == 0
    got, st = trajectories_resident(prog, 7, shots)
    assert st.cluster_span == 8 and st.launches == 1
    assert_cbits_match(got, want, st.boundary_draws)
    # shot offsets: shots [100, 164) of the same stream
    part, st2 = trajectories_resident(prog, 7, 64, shot0=100)
    want2, _, _ = orc.run_shots(prog, 7, 64, shot0=100)
    assert_cbits_match(part, want2, st2.boundary_draws)


def test_trajectories_match_per_shot_engine(gpu):
    from dqsim_bosonic_b200.statevector import run_program

    prog = prog_of(shot_circuit(12, 50, seed=3))
    got, st = trajectories_resident(prog, 11, 16)
    state = nat.State(12, 0)
    for i in range(16):
        state.reset()
        cb, _ = run_program(state, prog, 11 + i, nat.SEM_SHOTS, nat.EXEC_PER_GATE)
        if st.boundary_draws == 0:
            assert (cb == got[i]).all()


def test_run_trajectories_tuner(gpu):
    prog = prog_of(_circuits.trajectory_circuit(14, 6, seed=2))
    tuner = TrajectoryTuner(trial_shots=32)
    bits, times, fusion = run_trajectories(prog, 5, 64, 0, want_times=True, tuner=tuner)
    want, _, _ = orc.run_shots(prog, 5, 64)
    assert_cbits_match(bits, want, 0 if (bits == want).all() else 64)
    assert len(times) == 64 and fusion >= 0.0
    key = (14, prog.ninst, 0)
    assert key in tuner.cache and len(tuner.timings[key]) >= 3


def test_ragged_batch_states_and_cbits(gpu):
    rng = np.random.default_rng(99)
    ns = [3, 9, 12, 13, 14, 15, 16, 17, 18, 10, 16, 11]
    progs, seeds = [], []
    for k, n in enumerate(ns):
        depth = int(rng.integers(5, 41))
        if k % 3 == 0:
            circ = shot_circuit(n, depth, seed=k)
        else:
            circ = _circuits.random_circuit(k, n, depth)
        progs.append(prog_of(circ))
        seeds.append(1000 + k)
    cbits, states, st = run_batch(progs, seeds, want_states=True)
    # 17 and 18 qubits: HBM items of the persistent launch when the sweep
    # planner represents every gate, otherwise one engine run each
    assert st.engine_items + st.hbm_items == 2
    for k, p in enumerate(progs):
        want_cb, rc, _ = orc.run_shots(p, seeds[k], 1)
        assert rc == 0
        if st.boundary_draws == 0:
            assert (cbits[k] == want_cb[0]).all(), k
        if p.cbit_space == 0:
            ref, _, rc2, _ = orc.run(p, 0)
            assert rc2 == 0
            assert np.max(np.abs(states[k] - ref)) < 1e-12, k
        else:
            assert abs(np.vdot(states[k], states[k]).real - 1.0) < 1e-12


def test_ragged_batch_is_one_launch(gpu):
    """Resident (<= 16 qubits) and HBM-resident (17..19 qubits) items of a
    ragged u3 + cx batch run in one persistent launch; every final state
    matches the oracle within 1e-12."""
    ns = [10, 11, 13, 14, 16, 17, 18, 19, 12, 15]
    rng = np.random.default_rng(5)
    progs = [prog_of(_circuits.brickwork_u3_cx(n, int(rng.integers(5, 16)), seed=40 + k))
             for k, n in enumerate(ns)]
    seeds = [7 + k for k in range(len(ns))]
    cbits, states, st = run_batch(progs, seeds, want_states=True)
    assert st.launches == 1 and st.engine_items == 0 and st.hbm_items == 3
    assert st.cluster_span == 8
    for k, p in enumerate(progs):
        ref, _, rc, _ = orc.run(p, 0)
        assert rc == 0
        assert np.max(np.abs(states[k] - ref)) < 1e-12, (k, ns[k])


def test_ragged_batch_hbm_item_with_swaps_and_x(gpu):
    """An HBM item whose sweeps relabel qubits (swap) and open with X gates:
    its state is put back in canonical order before it is copied out."""
    n = 18
    insts = [g("x", 3), g("x", 17), g("h", 0), g("swap", 0, 17), g("cx", 17, 5), g("swap", 2, 11),
             g("u3", 11, 0.3, 0.2, 0.1), g("cp", 4, 16, 0.7), g("h", 16)]
    progs = [prog_of(JsonCircuit(n, insts)), prog_of(_circuits.brickwork_u3_cx(12, 4, seed=3))]
    cbits, states, st = run_batch(progs, [1, 2], want_states=True)
    assert st.hbm_items == 1 and st.engine_items == 0
    for k, p in enumerate(progs):
        ref, _, rc, _ = orc.run(p, 0)
        assert rc == 0
        assert np.max(np.abs(states[k] - ref)) < 1e-12, k


def test_ragged_batch_partial_state_outputs(gpu):
    progs = [prog_of(_circuits.brickwork_u3_cx(n, 4, seed=n)) for n in (11, 17, 12)]
    _, states, st = run_batch(progs, [1, 2, 3], want_states=[1])
    assert states[0] is None and states[2] is None
    ref, _, _, _ = orc.run(progs[1], 0)
    assert np.max(np.abs(states[1] - ref)) < 1e-12


def test_unsupported_gate_reached(gpu):
    circ = JsonCircuit(5, [g("h", 0), _circuits.gate("mystery_gate", [0, 1])])
    prog = prog_of(circ)
    with pytest.raises(RuntimeError, match='Unsupported generic gate: "mystery_gate"'):
        trajectories_resident(prog, 1, 4)
    with pytest.raises(RuntimeError, match='batch item 1: Unsupported generic gate'):
        run_batch([prog_of(JsonCircuit(3, [g("h", 0)])), prog], [1, 2])


def test_rejects_bad_arguments(gpu):
    prog = prog_of(_circuits.random_circuit(1, 17, 5))
    with pytest.raises(ValueError):
        trajectories_resident(prog, 1, 4)  # 17 qubits do not fit a cluster
    prog = prog_of(_circuits.random_circuit(1, 14, 5))
    with pytest.raises(ValueError):
        trajectories_resident(prog, 1, 4, opts=_opts(256, 1, 0))  # needs 2 CTAs
    with pytest.raises(ValueError):
        trajectories_resident(prog, 1, 4, opts=_opts(100, 0, 0))


def test_graph_plan_replays_match(gpu):
    prog = prog_of(_circuits.trajectory_circuit(15, 6, seed=4))
    plan = TrajectoryPlan(prog, 96)
    for seed in (3, 1000, 3):
        got, st = plan.run(seed)
        want, st2 = trajectories_resident(prog, seed, 96)
        assert st.cluster_span == st2.cluster_span == 4
        if st.boundary_draws == 0 and st2.boundary_draws == 0:
            assert (got == want).all()
        assert st.kernel_ms > 0.0
    plan.release()
