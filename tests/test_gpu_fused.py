"""Fused tile-sweep execution against the oracle (needs a B200).

The fused path reorders floating-point work (gate matrices applied inside
shared-memory tiles, diagonal gates folded into lazily applied phase
products, swaps as relabelings), so amplitudes are held to the 1e-12
absolute tolerance of the statevector contract, and measured outcomes must
match except for draws within 1e-12 of p1 (reported by the engine).
"""
import math

import numpy as np
import pytest

import _oracle
from _circuits import (JsonCircuit, brickwork_u3_cx, cond, g, gate, hadamard_diagonal_circuit,
                       hea_ansatz, qft_with_x, random_circuit, trajectory_circuit)
from dqsim_bosonic_b200 import StatevectorSimulator
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
from dqsim_bosonic_b200.statevector import SimulationResult, run_program

pytestmark = pytest.mark.gpu

ATOL = 1e-12


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


def fused_run(prog, seed=0, init=None, width=0, max_cost=0, semantics=nat.SEM_SIMULATE):
    st = nat.State(prog.num_qubits, 0)
    if init is not None:
        st.upload(init)
    cbits, prof = run_program(st, prog, seed, semantics, nat.EXEC_FUSED, width, False, False,
                              max_cost)
    return st, cbits, prof


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("n,depth,seed", [(10, 300, 1), (11, 300, 2), (12, 400, 3), (13, 400, 4),
                                          (14, 400, 5), (16, 300, 6), (17, 200, 7)])
def test_random_circuits_fused(gpu, n, depth, seed):
    prog = prog_of(random_circuit(100 + seed, n, depth))
    init = random_state(n, seed)
    want, _, rc, _ = _oracle.run(prog, 0, init)
    assert rc == 0
    st, _, prof = fused_run(prog, 0, init)
    got = st.download()
    assert prof.sweeps >= 1
    assert np.max(np.abs(got - want)) < ATOL


@pytest.mark.parametrize("width", [9, 10, 11, 12])
@pytest.mark.parametrize("max_cost", [0, 6, 20])
def test_fusion_widths_and_budgets(gpu, width, max_cost):
    n = 15
    prog = prog_of(random_circuit(7 * width + max_cost, n, 250))
    init = random_state(n, width)
    want, _, _, _ = _oracle.run(prog, 0, init)
    st, _, prof = fused_run(prog, 0, init, width, max_cost)
    assert np.max(np.abs(st.download() - want)) < ATOL


@pytest.mark.parametrize("n", [10, 13, 16])
def test_qft_relabel_probabilities_and_state(gpu, n):
    c = qft_with_x(n, 5)
    prog = prog_of(c)
    want, _, _, _ = _oracle.run(prog, 0)
    st, _, prof = fused_run(prog)
    res = SimulationResult(st, n, {}, None)
    # marginals are computed through the relabeling, without moving data
    for qs in ([n - 1, 0], [3, 1, 2], list(range(n - 1, -1, -1))):
        assert np.max(np.abs(res.probability_array(qs) - _oracle.marginal(want, qs))) < ATOL
    assert np.max(np.abs(res.statevector - want)) < ATOL
    # QFT of a basis state: uniform distribution
    assert np.allclose(np.abs(want) ** 2, 2.0 ** -n, atol=1e-12)


def swap_heavy(n, seed, depth=200):
    rng = np.random.default_rng(seed)
    insts = []
    for _ in range(depth):
        k = rng.integers(8)
        a, b, c = rng.choice(n, size=3, replace=False).tolist()
        th = float(rng.uniform(-3, 3))
        if k == 0:
            insts.append(g("swap", a, b))
        elif k == 1:
            insts.append(g("cswap", a, b, c))
        elif k == 2:
            insts.append(g("u3", a, th, 0.3 * th, -th))
        elif k == 3:
            insts.append(g("cp", a, b, th))
        elif k == 4:
            insts.append(g("rzz", a, b, th))
        elif k == 5:
            insts.append(g("ccx", a, b, c))
        elif k == 6:
            insts.append(gate("remote_link_psi_minus", [a, b]))
        else:
            insts.append(g("rxx", a, b, th))
    return JsonCircuit(n, insts)


@pytest.mark.parametrize("n,seed", [(10, 1), (12, 2), (14, 3), (16, 4)])
def test_swap_relabeling(gpu, n, seed):
    prog = prog_of(swap_heavy(n, seed))
    init = random_state(n, seed)
    want, _, _, _ = _oracle.run(prog, 0, init)
    st, _, _ = fused_run(prog, 0, init)
    res = SimulationResult(st, n, {}, None)
    assert np.max(np.abs(res.probability_array([0, n - 1, 2]) - _oracle.marginal(want, [0, n - 1, 2]))) < ATOL
    # a per-gate primitive on the relabelled state, then the canonical download
    one = prog_of(JsonCircuit(n, [g("h", 1), g("cx", 0, n - 1)]))
    nat.check(nat.lib().dq_apply_inst(st.handle, nat.ptr(one.insts[0:1])))
    nat.check(nat.lib().dq_apply_inst(st.handle, nat.ptr(one.insts[1:2])))
    _oracle.run_inplace(one, 0, want)
    assert np.max(np.abs(st.download() - want)) < ATOL


def measured(n, seed, layers=8):
    rng = np.random.default_rng(seed)
    insts = []
    for layer in range(layers):
        for q in range(n):
            insts.append(g("u3", q, *rng.uniform(0, 2 * math.pi, 3).tolist()))
        for q in range(layer % 2, n - 1, 2):
            insts.append(g("cx", q, q + 1))
        insts.append(g("swap", 0, n - 1))
        insts.append(g("cp", 1, n - 2, 0.4))
        insts.append(g("measure", (3 * layer) % n, layer % 4))
        insts.append(cond(layer % 4, 1, 1, g("x", (layer + 1) % n)))
        insts.append(cond(0, 2, 1, g("rzz", 2, n - 1, 0.7)))
        if layer % 3 == 1:
            insts.append(g("reset", (layer + 5) % n))
    insts.append(g("measure", 2, 5))
    return JsonCircuit(n, insts, ncbits=6)


@pytest.mark.parametrize("n,seed", [(10, 0), (11, 1), (13, 2), (15, 3)])
def test_measure_reset_conditional_fused(gpu, n, seed):
    prog = prog_of(measured(n, seed))
    for rseed in (seed, 77 + seed):
        want, wcb, rc, _ = _oracle.run(prog, rseed)
        st, gcb, prof = fused_run(prog, rseed)
        if prof.boundary_draws:
            continue
        assert gcb.tolist() == wcb.tolist()
        assert np.max(np.abs(st.download() - want)) < ATOL


def test_shots_semantics_fused_match_oracle(gpu):
    prog = prog_of(trajectory_circuit(n=12, layers=6, seed=3))
    want, rc, _ = _oracle.run_shots(prog, 55, 24)
    assert rc == 0
    for s in range(24):
        st, cb, prof = fused_run(prog, 55 + s, semantics=nat.SEM_SHOTS)
        if prof.boundary_draws:
            continue
        assert cb.tolist() == want[s].tolist()


def test_hea_ansatz_fused(gpu):
    c, _ = hea_ansatz(14, 4, 5)
    prog = prog_of(c)
    want, _, _, _ = _oracle.run(prog, 0)
    st, _, _ = fused_run(prog)
    assert np.max(np.abs(st.download() - want)) < ATOL


def test_brickwork20_fused_full_size(gpu):
    c = brickwork_u3_cx(20, 20, 1234)
    prog = prog_of(c)
    _oracle.set_threads(8)
    want, _, _, _ = _oracle.run(prog, 0)
    res = StatevectorSimulator(seed=0, exec="fused").simulate(c)
    got = res.statevector
    assert np.max(np.abs(got - want)) < ATOL
    idx = res.sample_indices(10000, None, 7)
    widx = _oracle.sample(want, list(range(19, -1, -1)), 7, 10000)
    assert int(np.sum(idx != widx)) <= res.last_boundary_draws


def test_qft24_fused_vs_oracle(gpu):
    c = qft_with_x(24, 9)
    prog = prog_of(c)
    _oracle.set_threads(8)
    want, _, _, _ = _oracle.run(prog, 0)
    res = StatevectorSimulator(seed=0, exec="fused").simulate(c)
    top = list(range(23, 13, -1))
    assert np.max(np.abs(res.probability_array(top) - _oracle.marginal(want, top))) < ATOL
    assert np.max(np.abs(res.statevector - want)) < ATOL


def test_distributed_variant_fused(gpu):
    from _circuits import distributed_qft_variant

    c = distributed_qft_variant(6, 3)
    prog = prog_of(c)
    want, _, _, _ = _oracle.run(prog, 0)
    st, _, _ = fused_run(prog)
    assert np.max(np.abs(st.download() - want)) < ATOL


@pytest.mark.parametrize("n,layers,seed", [(12, 12, 1), (15, 10, 2), (18, 8, 3), (21, 6, 4)])
def test_hadamard_phases_with_diagonals(gpu, n, layers, seed):
    prog = prog_of(hadamard_diagonal_circuit(n, layers, seed))
    init = random_state(n, seed)
    want, _, rc, _ = _oracle.run(prog, 0, init)
    assert rc == 0
    st, _, prof = fused_run(prog, 0, init)
    assert prof.sweeps >= 1
    assert np.max(np.abs(st.download() - want)) < ATOL
