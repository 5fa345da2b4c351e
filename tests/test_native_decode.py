"""The library's circuit decoder (``dq_circuit_decode``) against the Python one.

``dq_circuit_decode`` turns ``model_dump_json()`` text straight into dq_inst /
dq_cond records (the serde decoding of src/types.rs:8-135 plus the host
encoding).  The contract: whenever it accepts a text, the records, register
widths, classical space and generic gate names equal what the Python
decoder + encoder produce for the same text, bit for bit; everything else it
declines, and ``decode_program`` then reports the Python decoder's error or
result.  No GPU is used.
"""
from __future__ import annotations

import json
import math
import random
import struct

import numpy as np
import pytest

import _circuits as C
from dqsim_bosonic_b200.circuit import (_decode_native, decode_circuit_json, decode_program,
                                        encode)


def _python(text: str):
    return encode(decode_circuit_json(text))


def _same(a, b) -> None:
    assert a.insts.dtype == b.insts.dtype
    assert a.insts.tobytes() == b.insts.tobytes()
    assert a.conds.tobytes() == b.conds.tobytes()
    assert (a.num_qubits, a.num_cbits, a.cbit_space) == (b.num_qubits, b.num_cbits, b.cbit_space)
    assert a.gate_names == b.gate_names


def _check_text(text: str) -> bool:
    """Native result equals the Python one whenever native accepts; returns
    whether it accepted."""
    nat = _decode_native(text)
    try:
        py = _python(text)
        py_err = None
    except Exception as e:  # noqa: BLE001 - any error the Python path raises
        py, py_err = None, e
    if nat is None:
        # declined: decode_program gives exactly the Python outcome
        if py_err is not None:
            with pytest.raises(type(py_err)) as info:
                decode_program(text)
            assert str(info.value) == str(py_err)
        else:
            _same(decode_program(text), py)
        return False
    assert py_err is None, f"native accepted a text the Python decoder rejects: {py_err}"
    _same(nat, py)
    return True


def _every_kind_circuit(seed: int) -> C.JsonCircuit:
    rng = np.random.default_rng(seed)
    n = 6
    insts = []
    for kind in C._FIELDS:
        if kind == "measure":
            insts.append(C.g("measure", int(rng.integers(n)), int(rng.integers(8))))
            continue
        if C.GATE_ARITY[kind] > n:
            continue
        insts.append(C.random_gate(rng, n, kind))
    insts += [
        {"kind": "barrier"},
        {"kind": "classical", "name": "noop"},
        C.gate("Remote_Link_Psi_Minus", [0, 1]),
        C.gate("remote_epr", [2, 3], [0.5]),
        C.gate("NONLOCAL_CZ", [1, 4]),
        C.gate("remote_barrier", [0, 1, 2]),
        C.gate("circuit-block7", [0, 1, 2, 3, 4, 5, 0, 1, 2, 3], [1.0, 2.0]),
        C.gate("mystery", [3, 2 ** 31 + 5], []),
        C.cond(0, 3, 5, C.g("x", 2)),
        C.cond(2, 4, 1, C.cond(0, 1, 1, C.g("rz", 1, 0.25))),
        C.cond(0, 0, 0, C.gate("remote_cx", [0, 5])),
        C.cond(60, 4, 3, {"kind": "barrier"}),
    ]
    return C.JsonCircuit(n, insts, qregs={"a": {"name": "a", "size": 4, "base": 0},
                                          "b": {"name": "b", "size": 2, "base": 4}},
                         cregs={"c": {"name": "c", "size": 8, "base": 0},
                                "d": {"name": "d", "size": 2, "base": 8}})


def test_workload_circuits_decode_identically():
    circuits = [C.qft_with_x(30, 1234), C.brickwork_u3_cx(20, 20, 1234),
                C.distributed_qft_variant(14, 1234), C.trajectory_circuit(16, 12, 7)]
    circuits += [C.random_circuit(s, 9, 60) for s in range(5)]
    circuits += list(C.ragged_batch(16, 99))
    for c in circuits:
        text = c.model_dump_json()
        nat = _decode_native(text)
        assert nat is not None
        _same(nat, _python(text))


def test_every_kind_generic_names_and_condition_chains():
    for seed in range(4):
        text = _every_kind_circuit(seed).model_dump_json()
        nat = _decode_native(text)
        assert nat is not None
        py = _python(text)
        _same(nat, py)
    assert nat.conds.shape[0] == 5
    assert nat.cbit_space == 64
    assert set(nat.gate_names.values()) >= {"remote_link_psi_minus", "nonlocal_cz", "mystery",
                                            "circuit-block7", "remote_cx"}


# ---- text forms: a writer that varies whitespace, key order, number spelling ----

_WS = [" ", "\t", "\n", "\r", "  \n\t"]


def _num(v, rng: random.Random) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, int):
        return str(v)
    r = rng.random()
    if v == int(v) and abs(v) < 1e15 and r < 0.2:
        return str(int(v))                      # an integer token for an f64 field
    if r < 0.4:
        return "%.17e" % v
    if r < 0.55:
        return ("%.25e" % v).replace("e", "E")  # more digits than needed
    return repr(v)


def _write(obj, rng: random.Random, register_map: bool = False) -> str:
    """``register_map``: the dict is a qregs / cregs map, whose every key is a
    register (no ignored keys there)."""
    w = lambda: rng.choice(_WS) if rng.random() < 0.3 else ""  # noqa: E731
    if isinstance(obj, dict):
        items = list(obj.items())
        rng.shuffle(items)
        if not register_map and rng.random() < 0.3:
            items.insert(rng.randrange(len(items) + 1),
                         ("x_extra", {"k": [1, -2.5e-3, None, True, False, "s\\\"é\t"], "n": {}}))
        body = ",".join(f"{w()}{json.dumps(k)}{w()}:{w()}{_write(v, rng, k in ('qregs', 'cregs'))}{w()}"
                        for k, v in items)
        return "{" + body + w() + "}"
    if isinstance(obj, list):
        return "[" + ",".join(w() + _write(x, rng) + w() for x in obj) + "]"
    if isinstance(obj, str):
        return json.dumps(obj, ensure_ascii=rng.random() < 0.5)
    if obj is None:
        return "null"
    return _num(obj, rng)


def test_text_forms_decode_identically():
    rng = random.Random(2024)
    accepted = 0
    total = 0
    for seed in range(40):
        base = _every_kind_circuit(seed) if seed % 2 else C.random_circuit(seed, 7, 25)
        d = base.to_dict()
        for _ in range(3):
            total += 1
            accepted += _check_text(rng.choice(_WS) + _write(d, rng) + rng.choice(_WS))
    # every form above is well formed: the native decoder takes all of them
    assert accepted == total


def test_numbers_convert_exactly():
    """f64 fields: the native conversion gives Python's float() bit for bit."""
    rng = random.Random(7)
    tokens = ["0", "-0", "-0.0", "5e-324", "2.2250738585072014e-308", "1.7976931348623157e308",
              "0.1000000000000000055511151231257827", "123456789012345678901234567890",
              "9007199254740993", "1E+2", "1e-5", "3.141592653589793238462643383279"]
    for _ in range(1500):
        x = struct.unpack("<d", struct.pack("<Q", rng.getrandbits(64)))[0]
        if math.isfinite(x):
            tokens.append(repr(x))
            tokens.append("%.20e" % x)
        digits = "".join(rng.choice("0123456789") for _ in range(rng.randint(1, 40)))
        tokens.append(f"{rng.choice(['', '-'])}0.{digits}e{rng.randint(-320, 300)}")
    accepted = 0
    for tok in tokens:
        text = ('{"qregs": {"q": {"name": "q", "size": 1, "base": 0}}, "instructions": '
                f'[{{"kind": "rx", "qubit": 0, "theta": {tok}}}]}}')
        nat = _decode_native(text)
        want = float(json.loads(tok))
        if nat is None:
            assert not math.isfinite(want) or want == 0.0 or abs(want) < 2.3e-308
            continue
        accepted += 1
        got = float(nat.insts["p"][0][0])
        assert struct.pack("<d", got) == struct.pack("<d", want), tok
        _same(nat, _python(text))
    assert accepted > 0.8 * len(tokens)


_Q = '"qregs": {"q": {"name": "q", "size": 3, "base": 0}}'
_BAD = [
    "",
    "{not json",
    "[]",
    '{"instructions": []}',
    '{' + _Q + '}',
    '{' + _Q + ', "instructions": [{"qubit": 0}]}',
    '{' + _Q + ', "instructions": [{"kind": "hh", "qubit": 0}]}',
    '{' + _Q + ', "instructions": [{"kind": 3, "qubit": 0}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 1.0}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 1e0}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": -1}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": true}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 01}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 18446744073709551616}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0, "theta": NaN}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0, "theta": -Infinity}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0, "theta": 1e999}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0, "theta": "1"}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 2147483648}]}',
    '{' + _Q + ', "instructions": [{"kind": "measure", "qubit": 0, "cbit": 67108864}]}',
    '{' + _Q + ', "instructions": [{"kind": "gate", "name": "remote_cz", "params": [], "qubits": [0]}]}',
    '{' + _Q + ', "instructions": [{"kind": "gate", "name": "g", "params": [true], "qubits": [0]}]}',
    '{' + _Q + ', "instructions": [{"kind": "conditional", "condition": {"creg_base": 0, '
    '"creg_size": 65, "creg_value": 0}, "op": {"kind": "x", "qubit": 0}}]}',
    '{' + _Q + ', "instructions": [{"kind": "conditional", "condition": {"creg_base": 0, '
    '"creg_size": 1}, "op": {"kind": "x", "qubit": 0}}]}',
    '{' + _Q + ', "instructions": [{"kind": "classical", "name": "a\\qb"}]}',
    '{' + _Q + ', "instructions": [{"kind": "classical", "name": "tab\there"}]}',
    '{' + _Q + ', "cregs": null, "instructions": []}',
    '{' + _Q + ', "instructions": []} x',
    '{"qregs": {"q": {"name": "q", "size": 3}}, "instructions": []}',
    # legal forms left to the Python decoder (same result as before)
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": -0}]}',
    '{' + _Q + ', "instructions": [{"kind": "h", "qubit": 0, "qubit": 1}]}',
    '{' + _Q + ', ' + _Q + ', "instructions": []}',
    '{' + _Q + ', "instructions": [{"kind": "gate", "name": "REMOTE_İ", "params": [], "qubits": [0]}]}',
    '{' + _Q + ', "instructions": [{"kind": "classical", "name": "\\ud800x"}]}',
    '{' + _Q + ', "instructions": [{"kind": "rx", "qubit": 0, "theta": 1e-400}]}',
]


@pytest.mark.parametrize("text", _BAD)
def test_declined_texts_keep_the_python_outcome(text):
    assert _decode_native(text) is None
    _check_text(text)


def test_unicode_escapes_in_names():
    for name in ["Remote_\\u0045PR", "\\ud83d\\ude00", "\\u00e9t\\u00e9", "a\\/b\\\\c\\\"d",
                 "remote_link_phi_plus"]:
        text = ('{' + _Q + ', "instructions": [{"kind": "gate", "name": "' + name +
                '", "params": [], "qubits": [0, 1]}, {"kind": "classical", "name": "' + name + '"}]}')
        _check_text(text)
    ok = _decode_native('{' + _Q + ', "instructions": [{"kind": "gate", "name": "Remote_\\u0045PR", '
                        '"params": [], "qubits": [0, 1]}]}')
    assert ok is not None and ok.gate_names == {0: "remote_epr"}
