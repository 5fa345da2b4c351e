"""The sharded statevector (dqsim_bosonic_b200.sharded) on CPU shards: the
orchestration (relabelling, flips, per-rank gate reduction, exchanges,
distributed measurement) against the oracle's single-state run of the same
program.  Shards run through the oracle; ranks are either held by one process
(LocalShards) or are gloo processes (world size 2 and 4).

Tolerances: amplitudes 1e-12 (different summation order of p1 and of phase
factors); classical bits exact."""
import os
import socket

import numpy as np
import pytest

import _circuits as C
import _oracle as orc
from _shard_cpu import CpuShard
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
from dqsim_bosonic_b200.sharded import LocalShards, ShardedStatevector


def mixed_program(seed: int, n: int, depth: int, ncb: int = 4):
    """Random gates of every kind, with measures, resets and conditional gates."""
    rng = np.random.default_rng(seed)
    ins = []
    for i in range(depth):
        u = rng.random()
        if u < 0.06:
            ins.append(C.g("measure", int(rng.integers(n)), int(rng.integers(ncb))))
        elif u < 0.09:
            ins.append(C.g("reset", int(rng.integers(n))))
        elif u < 0.14:
            ins.append(C.cond(int(rng.integers(ncb - 1)), 2, int(rng.integers(4)), C.random_gate(rng, n)))
        else:
            ins.append(C.random_gate(rng, n))
    c = C.JsonCircuit(n, ins, ncbits=ncb)
    return encode(decode_circuit_json(c.model_dump_json()))


def reduction_program(n: int = 7):
    """Gates that hit each per-rank reduction with qubits n-1, n-2 global."""
    a, b = n - 1, n - 2
    G = C.g
    ins = [G("h", 0), G("h", 1), G("h", 2), G("ry", 3, 0.7),
           G("x", a), G("y", b), G("z", a), G("s", b), G("t", a), G("rz", b, 0.3), G("p", a, 1.1),
           G("cx", a, 0), G("cy", b, 1), G("cz", 0, a), G("cp", 1, b, 0.4), G("cp", a, b, 0.9),
           G("crz", 2, a, 0.5), G("crz", a, b, 1.3), G("rzz", 0, b, 0.8), G("rzz", a, b, 0.2),
           G("cu", a, 1, 0.3, 0.2, 0.1, 0.6), G("cu3", b, 2, 0.5, 0.4, 0.3), G("ccx", a, b, 0),
           G("cswap", a, 0, 1), G("swap", 0, a), G("h", a), G("cx", 0, b), G("crx", 1, a, 0.4),
           G("c3x", a, b, 0, 1), G("rccx", a, 0, 1), G("c3sqrtx", a, 0, 1, 2), G("c4x", b, 0, 1, 2, a),
           G("rxx", b, 3, 0.7), C.gate("nonlocal_cz", [a, 2]), C.gate("remote_cx", [b, 3]),
           C.gate("remote_link_psi_minus", [a, b]), G("u3", b, 0.2, 0.3, 0.4),
           G("measure", a, 0), G("reset", b), C.cond(0, 1, 1, G("x", a)), G("sx", a),
           G("measure", b, 1)]
    c = C.JsonCircuit(n, ins, ncbits=2)
    return encode(decode_circuit_json(c.model_dump_json()))


def run_local(prog, world, seed, n=None):
    sv = ShardedStatevector(n or prog.num_qubits, LocalShards(world), backend=lambda nl, r: CpuShard(nl, r),
                            chunk=1 << 3)
    cb = sv.run(prog, seed)
    return sv, cb


@pytest.mark.parametrize("world", [2, 4, 8])
def test_reduction_rules_match_the_oracle(world):
    prog = reduction_program(7)
    want, wcb, rc, _ = orc.run(prog, 11)
    assert rc == 0
    sv, cb = run_local(prog, world, 11)
    assert np.array_equal(cb, wcb)
    assert np.max(np.abs(sv.statevector() - want)) < 1e-12
    assert sv.exchanges > 0


@pytest.mark.parametrize("world,seed", [(2, 1), (4, 2), (8, 3), (4, 4)])
def test_random_programs_match_the_oracle(world, seed):
    prog = mixed_program(seed, 9, 160)
    want, wcb, rc, _ = orc.run(prog, 100 + seed)
    assert rc == 0
    sv, cb = run_local(prog, world, 100 + seed)
    assert np.array_equal(cb, wcb)
    assert np.max(np.abs(sv.statevector() - want)) < 1e-12
    for qs in ([8, 0, 3], [7], [1, 8, 2, 7]):
        assert np.max(np.abs(sv.probabilities(qs) - orc.marginal(want, qs))) < 1e-12


def test_rejects_bad_geometry():
    with pytest.raises(ValueError):
        ShardedStatevector(4, LocalShards(3), backend=lambda nl, r: CpuShard(nl, r))
    with pytest.raises(ValueError):
        ShardedStatevector(2, LocalShards(4), backend=lambda nl, r: CpuShard(nl, r))


def test_unsupported_generic_gate_raises_like_simulate():
    c = C.JsonCircuit(5, [C.g("h", 4), C.gate("frobnicate", [4, 0])])
    prog = encode(decode_circuit_json(c.model_dump_json()))
    sv = ShardedStatevector(5, LocalShards(2), backend=lambda nl, r: CpuShard(nl, r))
    with pytest.raises(NotImplementedError, match="Unsupported generic gate"):
        sv.run(prog, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, seed, out_dir):
    import sys

    sys.path.insert(0, os.path.dirname(__file__))
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        prog = mixed_program(seed, 9, 160)
        sv = ShardedStatevector(9, None, backend=lambda nl, r: CpuShard(nl, r), chunk=1 << 4)
        cb = sv.run(prog, 200 + seed)
        v = sv.statevector()
        p = sv.probabilities([8, 0, 5])
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), cb=cb, v=v, p=p, ex=sv.exchanges)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_gloo_ranks_match_the_oracle(world, tmp_path):
    import torch.multiprocessing as mp

    seed = 7 + world
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, seed, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    prog = mixed_program(seed, 9, 160)
    want, wcb, rc, _ = orc.run(prog, 200 + seed)
    for r in range(world):
        d = np.load(tmp_path / f"r{r}.npz")
        assert np.array_equal(d["cb"], wcb)
        assert np.max(np.abs(d["v"] - want)) < 1e-12
        assert np.max(np.abs(d["p"] - orc.marginal(want, [8, 0, 5]))) < 1e-12
        assert int(d["ex"]) > 0
