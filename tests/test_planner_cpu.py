"""The fused-sweep planner and encoder on the CPU (no GPU).

dq_debug_plan runs the real planner/encoder of the engine and returns the
encoded sweep programs; tests/_sweep_emu.py executes them like the kernel
does.  The result must match the oracle within the fused path's 1e-12
amplitude tolerance.
"""
import numpy as np
import pytest

import _oracle
from _circuits import (JsonCircuit, brickwork_u3_cx, g, gate, hadamard_diagonal_circuit, hea_ansatz,
                       hea_param_circuit, qft_with_x, random_circuit)
from _sweep_emu import canonical, emulate
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import decode_circuit_json, encode

ATOL = 1e-12


def prog_of(c):
    return encode(decode_circuit_json(c.model_dump_json()))


def random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def check(c, seed=0, opts=None):
    prog = prog_of(c)
    n = prog.num_qubits
    init = random_state(n, seed)
    want, _, rc, _ = _oracle.run(prog, 0, init)
    assert rc == 0
    got, perm, ns = emulate(prog, init, opts)
    got = canonical(got, perm)
    err = np.max(np.abs(got - want))
    assert err < ATOL, f"max error {err} over {ns} sweeps"
    return ns


@pytest.mark.parametrize("n,depth,seed", [(10, 120, 1), (11, 120, 2), (12, 150, 3), (13, 150, 4),
                                          (14, 120, 5)])
def test_random_circuits_planned(engine_lib, n, depth, seed):
    check(random_circuit(200 + seed, n, depth), seed)


@pytest.mark.parametrize("width", [10, 11, 12])
@pytest.mark.parametrize("max_cost", [0, 6, 30])
def test_widths_and_budgets_planned(engine_lib, width, max_cost):
    opts = nat.RunOpts(0, nat.EXEC_FUSED, width, 0, 0, max_cost)
    check(random_circuit(31 * width + max_cost, 13, 120), width, opts)


@pytest.mark.parametrize("n", [10, 12, 14])
def test_qft_planned(engine_lib, n):
    ns = check(qft_with_x(n, 3))
    assert ns >= 1


def test_hea_planned(engine_lib):
    c, _ = hea_ansatz(13, 3, 4)
    check(c)


def test_brickwork_planned(engine_lib):
    check(brickwork_u3_cx(13, 8, 2))


def test_single_gate_kinds_planned(engine_lib):
    n = 12
    rng = np.random.default_rng(9)
    from _circuits import UNITARY_KINDS, random_gate

    for kind in UNITARY_KINDS:
        if kind in ("u0",):
            continue
        insts = [random_gate(rng, n, kind) for _ in range(6)]
        check(JsonCircuit(n, insts), 3)


def test_remote_and_swap_planned(engine_lib):
    n = 12
    insts = [g("h", q) for q in range(n)]
    insts += [gate("remote_link_psi_minus", [3, 9]), g("swap", 0, 11), g("cswap", 2, 5, 10),
              gate("nonlocal_cz", [1, 7]), g("rxx", 4, 8, 0.3), gate("remote_link_phi_plus", [6, 0]),
              g("swap", 3, 4), g("cp", 11, 0, 0.9), g("rzz", 5, 6, 1.1)]
    check(JsonCircuit(n, insts), 2)


def test_leading_x_gates_fold_into_the_load():
    """X gates that open a register phase cost nothing: they become a flip of
    the phase's load address.  X after other ops on its qubit must stay an op."""
    import struct

    from _sweep_emu import plan

    prog = prog_of(qft_with_x(12, 3))
    blobs, _, _, _ = plan(prog)
    m, rb, nphase, _ = struct.unpack_from("<4I", blobs[0], 0)
    off_phase = struct.unpack_from("<I", blobs[0], 64)[0]
    tile_xload = struct.unpack_from("<I", blobs[0], 88)[0]
    xloads = [struct.unpack_from("<I", blobs[0], off_phase + 192 * p + 184)[0] for p in range(nphase)]
    assert tile_xload or any(xloads), "no X gate was folded"
    # X before and after other gates on the same qubits, controls included
    insts = []
    for q in range(12):
        insts += [g("x", q), g("h", q), g("x", q), g("ry", q, 0.3 + q), g("x", q)]
    insts += [g("cx", 0, 5), g("x", 5), g("x", 0), g("cp", 3, 7, 0.7), g("x", 7)]
    check(JsonCircuit(12, insts), seed=4)
    check(JsonCircuit(12, insts[::-1]), seed=5)


def _plan_ops(prog):
    """(sweep header flags, [(type, b0, b1, flags) per op]) of every planned sweep."""
    import struct

    from _sweep_emu import plan

    blobs, _, _, _ = plan(prog)
    out = []
    for b in blobs:
        off_op = struct.unpack_from("<I", b, 68)[0]
        hflags = struct.unpack_from("<I", b, 104)[0]
        nph = struct.unpack_from("<I", b, 8)[0]
        off_phase = struct.unpack_from("<I", b, 64)[0]
        ops = []
        for p in range(nph):
            ob, oe = struct.unpack_from("<2I", b, off_phase + p * 192 + 176)
            for o in range(ob, oe):
                w0, w1 = struct.unpack_from("<2I", b, off_op + 32 * o)
                ops.append((w0 & 0xFF, (w0 >> 8) & 0xFF, (w0 >> 16) & 0xFF, (w1 >> 8) & 0xFF))
        out.append((hflags, ops))
    return out


def test_hadamard_phases_are_marked(engine_lib):
    # QFT: every phase of every sweep is an H phase (the H-only kernel build); the cp
    # phases of a target whose partners on register bits are all below it get FL_LOWF
    # tables (2^b products), the others (lower qubits on higher register bits) full ones
    sweeps = _plan_ops(prog_of(qft_with_x(14, 3)))
    assert all(fl & 1 for fl, _ in sweeps)
    subs = [op for _, ops in sweeps for op in ops if op[0] == 7 and op[3] & 6 == 6]
    assert any(op[3] & 8 for op in subs) and any(not op[3] & 8 for op in subs)
    # an H phase's ops sit on register bits 0..K-1 in order right after the marker
    for _, ops in sweeps:
        for i, op in enumerate(ops):
            if op[0] == 9:
                k = op[2]
                assert [o[1] for o in ops[i + 1:i + 1 + k]] == list(range(k))
    # pending phases on higher qubits: H phases whose flush tables need every register bit
    sweeps = _plan_ops(prog_of(hadamard_diagonal_circuit(15, 10, 2)))
    subs = [op for _, ops in sweeps for op in ops if op[0] == 7 and op[3] & 6 == 6]
    assert any(op[3] & 8 == 0 for op in subs)
    assert any(op[0] == 9 for _, ops in sweeps for op in ops)


@pytest.mark.parametrize("n,layers,seed", [(12, 12, 1), (14, 10, 2)])
def test_hadamard_diagonal_circuits_planned(engine_lib, n, layers, seed):
    check(hadamard_diagonal_circuit(n, layers, seed), seed)


def test_sweep_builds_chosen_per_workload(engine_lib):
    # header flags pick the kernel build: QFT sweeps are all Hadamard straight-line
    # phases (SWF_HONLY = 1), u3 + cx brickwork sweeps plain one-qubit ops (SWF_UONLY = 2),
    # the HEA forward pass real-2x2 straight-line phases (SWF_RONLY = 4) except its last
    # sweep, which also carries the final phase flushes
    import struct

    from _sweep_emu import plan

    def flags(prog):
        blobs, _, _, _ = plan(prog)
        return [struct.unpack_from("<I", b, 104)[0] for b in blobs], \
               [struct.unpack_from("<I", b, 108)[0] for b in blobs]

    f, g = flags(prog_of(qft_with_x(20, 3)))
    assert f and all(x == 1 for x in f)
    assert any(g)  # some sweeps' last phase writes straight to the state
    f, g = flags(prog_of(brickwork_u3_cx(20, 6, 1)))
    assert f and all(x == 2 for x in f) and any(g)
    c, theta, _ = hea_param_circuit(16, 4, seed=1)

    class P:
        pass

    p = P()
    p.insts = c.bind(np.asarray(theta))
    p.num_qubits, p.ninst = 16, len(p.insts)
    f, _ = flags(p)
    assert f[:-1] and all(x == 4 for x in f[:-1])
