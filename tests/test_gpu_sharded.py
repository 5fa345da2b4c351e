"""The sharded statevector on one GPU: 2 and 4 ranks held by one process
(LocalShards), each shard an engine state (NativeShard), against the
single-state engine and the oracle.  No collective library is involved (this
run has one GPU); the gloo tests cover the one-process-per-rank path.

Tolerance: amplitudes 1e-12 (fused tiles, different phase-factor order)."""
import numpy as np
import pytest

import _circuits as C
import _oracle as orc
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
from dqsim_bosonic_b200.sharded import LocalShards, NativeShard, ShardedStatevector
from dqsim_bosonic_b200.statevector import run_program
from test_sharded_cpu import mixed_program, reduction_program

pytestmark = pytest.mark.gpu


def single(prog, seed):
    st = nat.State(prog.num_qubits, 0)
    cb, _ = run_program(st, prog, seed, nat.SEM_SIMULATE, nat.EXEC_FUSED)
    v = st.download()
    st.release()
    return v, cb


@pytest.mark.parametrize("world", [2, 4])
def test_reduction_rules_on_gpu_shards(gpu, world):
    prog = reduction_program(9)
    want, wcb, rc, _ = orc.run(prog, 3)
    assert rc == 0
    sv = ShardedStatevector(9, LocalShards(world), device=0)
    cb = sv.run(prog, 3)
    assert np.array_equal(cb, wcb)
    assert np.max(np.abs(sv.statevector() - want)) < 1e-12
    sv.release()


@pytest.mark.parametrize("n,world,seed", [(12, 2, 1), (12, 4, 2), (14, 4, 3)])
def test_mixed_programs_on_gpu_shards(gpu, n, world, seed):
    prog = mixed_program(seed, n, 300)
    want, wcb = single(prog, 50 + seed)
    sv = ShardedStatevector(n, LocalShards(world), device=0, chunk=1 << 8)
    cb = sv.run(prog, 50 + seed)
    assert np.array_equal(cb, wcb)
    assert np.max(np.abs(sv.statevector() - want)) < 1e-12
    qs = [n - 1, 0, n - 2, 3]
    assert np.max(np.abs(sv.probabilities(qs) - orc.marginal(want, qs))) < 1e-12
    assert sv.exchanges > 0
    sv.release()


def test_qft20_over_four_shards(gpu):
    c = C.qft_with_x(20, 1234)
    prog = encode(decode_circuit_json(c.model_dump_json()))
    want, _ = single(prog, 0)
    sv = ShardedStatevector(20, LocalShards(4), device=0)
    sv.run(prog, 0)
    assert np.max(np.abs(sv.statevector() - want)) < 1e-12
    p = sv.probabilities(list(range(19, 9, -1)))
    assert abs(p.sum() - 1.0) < 1e-12
    sv.release()
