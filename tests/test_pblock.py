"""The p-block merge (merge_blocks, src/distributed/pblock/model.rs:35-57).

CPU: the oracle's merge against an independent construction (the Kronecker
product of the two states, reordered to the merged qubit order), exact.
GPU: dq_block_merge against the oracle, bit-identical (the merge is one
num-complex multiplication per amplitude), and its argument checks."""
import ctypes

import numpy as np
import pytest

import _oracle as orc
from dqsim_bosonic_b200 import _native as nat


def rand_state(n, rng):
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def kron_merge(a, qa, b, qb):
    """psi_a (x) psi_b as a tensor over the merged ascending qubits."""
    u = sorted(set(qa) | set(qb))
    n = len(u)
    out = np.zeros(1 << n, dtype=np.complex128)
    for i in range(1 << n):
        la = sum(((i >> u.index(q)) & 1) << k for k, q in enumerate(qa))
        lb = sum(((i >> u.index(q)) & 1) << k for k, q in enumerate(qb))
        out[i] = a[la] * b[lb]
    return out, u


CASES = [([0, 1, 2], [3, 4]), ([5, 9], [0, 3, 7]), ([1, 4, 6, 8], [2]), ([0, 2, 4, 6], [1, 3, 5, 7])]


@pytest.mark.parametrize("qa,qb", CASES)
def test_oracle_merge_is_the_reordered_kronecker_product(qa, qb):
    rng = np.random.default_rng(len(qa) * 10 + len(qb))
    a, b = rand_state(len(qa), rng), rand_state(len(qb), rng)
    got, u = orc.block_merge(a, qa, b, qb)
    want, wu = kron_merge(a, qa, b, qb)
    assert u == wu
    assert np.array_equal(got, want)


def test_kronecker_identity_for_adjacent_blocks():
    # blocks on qubits [0..k) and [k..n): the merged state is kron(b, a)
    rng = np.random.default_rng(3)
    a, b = rand_state(3, rng), rand_state(4, rng)
    got, _ = orc.block_merge(a, [0, 1, 2], b, [3, 4, 5, 6])
    assert np.allclose(got, np.kron(b, a), atol=0, rtol=1e-15)


def _gpu_merge(a, qa, b, qb, nout=None):
    sa, sb = nat.State(len(qa), 0), nat.State(len(qb), 0)
    sa.upload(a)
    sb.upload(b)
    u = sorted(set(qa) | set(qb))
    out = nat.State(len(u) if nout is None else nout, 0)
    qa_ = np.asarray(qa, dtype=np.uint32)
    qb_ = np.asarray(qb, dtype=np.uint32)
    rc = nat.lib().dq_block_merge(sa.handle, nat.ptr(qa_), qa_.size, sb.handle, nat.ptr(qb_), qb_.size,
                                  out.handle)
    v = out.download() if rc == 0 else None
    for s in (sa, sb, out):
        s.release()
    return rc, v, u


@pytest.mark.gpu
@pytest.mark.parametrize("qa,qb", CASES + [(list(range(0, 20, 2)), list(range(1, 20, 2))),
                                           (list(range(12)), list(range(12, 22)))])
def test_gpu_merge_matches_the_oracle_bit_for_bit(gpu, qa, qb):
    rng = np.random.default_rng(sum(qa) + 7 * sum(qb))
    a, b = rand_state(len(qa), rng), rand_state(len(qb), rng)
    rc, got, u = _gpu_merge(a, qa, b, qb)
    assert rc == 0
    want, wu = orc.block_merge(a, qa, b, qb)
    assert u == wu
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gpu_merge_through_the_block_api_after_gates(gpu):
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from dqsim_bosonic_b200.pblock import Block, merge_blocks
    from dqsim_bosonic_b200.statevector import run_program
    import _circuits as C

    a = Block([7, 2, 5])          # sorted to [2, 5, 7]
    b = Block([0, 9])
    assert a.qubits == [2, 5, 7] and a.local(7) == 2
    with pytest.raises(ValueError):
        a.local(4)
    pa = encode(decode_circuit_json(C.random_circuit(1, 3, 30).model_dump_json()))
    pb = encode(decode_circuit_json(C.random_circuit(2, 2, 20).model_dump_json()))
    run_program(a.state, pa, 0, nat.SEM_SIMULATE, nat.EXEC_PER_GATE)
    run_program(b.state, pb, 0, nat.SEM_SIMULATE, nat.EXEC_PER_GATE)
    m = merge_blocks(a, b)
    assert m.qubits == [0, 2, 5, 7, 9]
    want, _ = orc.block_merge(a.statevector(), a.qubits, b.statevector(), b.qubits)
    assert np.array_equal(m.statevector(), want)
    for blk in (a, b, m):
        blk.release()


@pytest.mark.gpu
def test_gpu_merge_rejects_bad_arguments(gpu):
    rng = np.random.default_rng(0)
    a, b = rand_state(2, rng), rand_state(2, rng)
    rc, _, _ = _gpu_merge(a, [3, 1], b, [0, 2])          # not ascending
    assert rc == nat.DQ_ERR_INVALID_ARG
    rc, _, _ = _gpu_merge(a, [0, 1], b, [2, 3], nout=5)  # wrong merged size
    assert rc == nat.DQ_ERR_INVALID_ARG
    assert b"merged state" in nat.lib().dq_last_error()
    rc, v, u = _gpu_merge(a, [0, 1], b, [1, 2])          # a shared qubit takes one position
    want, wu = orc.block_merge(a, [0, 1], b, [1, 2])
    assert rc == 0 and u == wu == [0, 1, 2] and np.array_equal(v, want)
