"""A reset / set_basis state is written lazily: the first fused sweep of the
next run generates its tiles from the basis index instead of reading memory,
and every other consumer writes the basis vector first.  Each path against
the oracle from the same basis state.  Tolerance: fused runs 1e-12
(amplitudes), exact paths bit-identical."""
import ctypes

import numpy as np
import pytest

import _circuits as C
import _oracle as orc
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
from dqsim_bosonic_b200.statevector import run_program

pytestmark = pytest.mark.gpu


def prog_of(ins, n, ncb=0):
    return encode(decode_circuit_json(C.JsonCircuit(n, ins, ncbits=ncb).model_dump_json()))


def basis(n, k):
    v = np.zeros(1 << n, dtype=np.complex128)
    v[k] = 1.0
    return v


@pytest.mark.parametrize("k", [0, 1, 0b10110011101011, (1 << 14) - 1])
def test_fused_run_from_a_lazy_basis_state(gpu, k):
    n = 14
    prog = encode(decode_circuit_json(C.random_circuit(5, n, 200).model_dump_json()))
    st = nat.State(n, 0)
    st.set_basis(k)
    _, prof = run_program(st, prog, 0, nat.SEM_SIMULATE, nat.EXEC_FUSED)
    assert prof.sweeps > 0
    want = orc.run_unitary(prog.insts, n, init=basis(n, k))
    assert np.max(np.abs(st.download() - want)) < 1e-12


def test_leading_x_gates_fold_into_a_synthesised_first_sweep(gpu):
    n = 16
    prog = encode(decode_circuit_json(C.qft_with_x(n, 99).model_dump_json()))
    st = nat.State(n, 0)
    k = 0b1011001110001101
    st.set_basis(k)
    run_program(st, prog, 0, nat.SEM_SIMULATE, nat.EXEC_FUSED)
    want = orc.run_unitary(prog.insts, n, init=basis(n, k))
    assert np.max(np.abs(st.download() - want)) < 1e-12


def test_measure_first_and_per_gate_runs_write_the_basis_first(gpu):
    n = 12
    k = 0b100101101001
    ins = [C.g("measure", 3, 0), C.g("h", 3), C.g("measure", 0, 1), C.g("cx", 0, 5), C.g("h", 11)]
    prog = prog_of(ins, n, 2)
    for mode in (nat.EXEC_FUSED, nat.EXEC_PER_GATE):
        st = nat.State(n, 0)
        st.set_basis(k)
        cb, _ = run_program(st, prog, 4, nat.SEM_SIMULATE, mode)
        want, wcb, rc, _ = orc.run(prog, 4, init=basis(n, k))
        assert rc == 0 and np.array_equal(cb, wcb)
        assert np.array_equal(st.download(), want)


def test_relabel_only_run_keeps_the_pending_basis(gpu):
    n = 12
    k = 0b000000000101
    prog = prog_of([C.g("swap", 0, 9), C.g("swap", 2, 11)], n)
    st = nat.State(n, 0)
    st.set_basis(k)
    run_program(st, prog, 0, nat.SEM_SIMULATE, nat.EXEC_FUSED)
    want = orc.run_unitary(prog.insts, n, init=basis(n, k))
    assert np.array_equal(st.download(), want)


def test_queries_copy_and_upload_see_the_basis_state(gpu):
    n = 12
    k = 1234
    st = nat.State(n, 0)
    st.set_basis(k)
    p = ctypes.c_double()
    nat.check(nat.lib().dq_measure_p1(st.handle, 4, ctypes.byref(p)))
    assert p.value == float((k >> 4) & 1)
    st.set_basis(k)
    other = nat.State(n, 0)
    nat.check(nat.lib().dq_state_copy(other.handle, st.handle))
    assert np.array_equal(other.download(), basis(n, k))
    fresh = nat.State(n, 0)                 # created lazily as |0>
    assert np.array_equal(fresh.download(), basis(n, 0))
    v = np.random.default_rng(1).normal(size=1 << n) + 0j
    fresh.set_basis(7)
    fresh.upload(v)                          # an upload replaces the pending basis
    assert np.array_equal(fresh.download(), v)
    for s in (st, other, fresh):
        s.release()
