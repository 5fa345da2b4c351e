"""Circuit decoding and encoding for the statevector engine.

The reference hands its Rust core one JSON string per circuit, produced by
``circuit.model_dump_json()`` and decoded by serde into the structs of
``src/types.rs:8-135``.  This module restates that decoding (same variant
tags, field names, required fields, ignored extra fields and defaults) and
encodes each decoded instruction into the POD ``dq_inst`` records that the
C ABI takes.

serde rules restated here:
  * ``Circuit``: ``qregs`` (map of ``Register``) and ``instructions`` are
    required; ``cregs`` defaults to an empty map; unknown keys are ignored.
  * ``Register``: ``name``, ``size``, ``base`` required.
  * ``Instruction``: internally tagged by ``kind`` (snake_case variant name);
    every listed field is required; ``usize`` fields reject floats, bools and
    negatives; ``f64`` fields accept JSON integers and floats.
  * ``num_qubits`` / ``num_cbits`` = max(base + size) over the registers
    (0 when there are none), ``types.rs:24-38``.
"""
from __future__ import annotations

import ctypes
import json
import math
import struct
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from ._native import COND_DTYPE, INST_DTYPE, KIND, MAX_INST_QUBITS

# variant tag -> ordered (field name, type) list; "u" = usize, "f" = f64
_FIELDS: dict[str, list[tuple[str, str]]] = {}
for _k in ("id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "u0", "reset"):
    _FIELDS[_k] = [("qubit", "u")]
_FIELDS.update(
    {
        "u3": [("qubit", "u"), ("theta", "f"), ("phi", "f"), ("lam", "f")],
        "u": [("qubit", "u"), ("theta", "f"), ("phi", "f"), ("lam", "f")],
        "u2": [("qubit", "u"), ("phi", "f"), ("lam", "f")],
        "u1": [("qubit", "u"), ("lam", "f")],
        "p": [("qubit", "u"), ("lam", "f")],
        "rx": [("qubit", "u"), ("theta", "f")],
        "ry": [("qubit", "u"), ("theta", "f")],
        "rz": [("qubit", "u"), ("phi", "f")],
        "cx": [("control", "u"), ("target", "u")],
        "cz": [("control", "u"), ("target", "u")],
        "cy": [("control", "u"), ("target", "u")],
        "ch": [("control", "u"), ("target", "u")],
        "csx": [("control", "u"), ("target", "u")],
        "swap": [("a", "u"), ("b", "u")],
        "crx": [("control", "u"), ("target", "u"), ("theta", "f")],
        "cry": [("control", "u"), ("target", "u"), ("theta", "f")],
        "crz": [("control", "u"), ("target", "u"), ("lam", "f")],
        "cu1": [("control", "u"), ("target", "u"), ("lam", "f")],
        "cp": [("control", "u"), ("target", "u"), ("lam", "f")],
        "cu3": [("control", "u"), ("target", "u"), ("theta", "f"), ("phi", "f"), ("lam", "f")],
        "cu": [("control", "u"), ("target", "u"), ("theta", "f"), ("phi", "f"), ("lam", "f"),
               ("gamma", "f")],
        "rxx": [("a", "u"), ("b", "u"), ("theta", "f")],
        "rzz": [("a", "u"), ("b", "u"), ("theta", "f")],
        "ccx": [("control1", "u"), ("control2", "u"), ("target", "u")],
        "rccx": [("control1", "u"), ("control2", "u"), ("target", "u")],
        "cswap": [("control", "u"), ("target1", "u"), ("target2", "u")],
        "rc3x": [("control1", "u"), ("control2", "u"), ("control3", "u"), ("target", "u")],
        "c3x": [("control1", "u"), ("control2", "u"), ("control3", "u"), ("target", "u")],
        "c3sqrtx": [("control1", "u"), ("control2", "u"), ("control3", "u"), ("target", "u")],
        "c4x": [("control1", "u"), ("control2", "u"), ("control3", "u"), ("control4", "u"),
                ("target", "u")],
        "measure": [("qubit", "u"), ("cbit", "u")],
        "barrier": [],
        "classical": [("name", "s")],
        "gate": [("name", "s"), ("params", "fl"), ("qubits", "ul")],
        "conditional": [("condition", "cond"), ("op", "inst")],
    }
)

# Generic `gate` names understood by the dispatcher
# (statevector/simulator.rs:571-600 and 802-831), matched after to_lowercase().
_GENERIC = {
    "remote_link_phi_plus": "g_phi_plus",
    "remote_epr": "g_phi_plus",
    "remote_link_psi_minus": "g_psi_minus",
    "remote_link_psi_plus": "g_psi_plus",
    "nonlocal_cz": "g_cz",
    "remote_cz": "g_cz",
    "remote_cx": "g_cx",
    "remote_barrier": "g_noop",
    "remote_cu1": "g_noop",
}

_U64_MAX = (1 << 64) - 1


class CircuitDecodeError(ValueError):
    """JSON that serde would reject for the reference's Circuit type."""


def _usize(v: Any, where: str) -> int:
    if isinstance(v, bool) or not isinstance(v, int):
        raise CircuitDecodeError(f"invalid type for {where}: expected usize, got {v!r}")
    if v < 0 or v > _U64_MAX:
        raise CircuitDecodeError(f"invalid value for {where}: {v} is not a usize")
    return v


def _f64(v: Any, where: str) -> float:
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        raise CircuitDecodeError(f"invalid type for {where}: expected f64, got {v!r}")
    f = float(v)
    if not math.isfinite(f):
        raise CircuitDecodeError(f"invalid value for {where}: {v!r}")
    return f


def _string(v: Any, where: str) -> str:
    if not isinstance(v, str):
        raise CircuitDecodeError(f"invalid type for {where}: expected string, got {v!r}")
    return v


@dataclass
class Instruction:
    """One decoded ``Instruction`` (src/types.rs:60-135)."""

    kind: str
    fields: dict[str, Any]
    condition: tuple[int, int, int] | None = None  # (creg_base, creg_size, creg_value)
    op: "Instruction | None" = None

    def qubits(self) -> list[int]:
        """``Instruction::qubits`` (src/types.rs:348-418)."""
        if self.kind == "conditional":
            return self.op.qubits()
        if self.kind in ("barrier", "classical"):
            return []
        if self.kind == "gate":
            return list(self.fields["qubits"])
        return [self.fields[n] for n, t in _FIELDS[self.kind] if t == "u" and n != "cbit"]


@dataclass
class Register:
    name: str
    size: int
    base: int


@dataclass
class Circuit:
    """A decoded ``Circuit`` (src/types.rs:15-39)."""

    qregs: dict[str, Register]
    cregs: dict[str, Register]
    instructions: list[Instruction] = field(default_factory=list)

    def num_qubits(self) -> int:
        return max((r.base + r.size for r in self.qregs.values()), default=0)

    def num_cbits(self) -> int:
        return max((r.base + r.size for r in self.cregs.values()), default=0)


def _decode_register(v: Any, where: str) -> Register:
    if not isinstance(v, dict):
        raise CircuitDecodeError(f"invalid type for {where}: expected struct Register")
    for f in ("name", "size", "base"):
        if f not in v:
            raise CircuitDecodeError(f"missing field `{f}` in {where}")
    return Register(_string(v["name"], where + ".name"), _usize(v["size"], where + ".size"),
                    _usize(v["base"], where + ".base"))


def _decode_registers(v: Any, where: str) -> dict[str, Register]:
    if not isinstance(v, dict):
        raise CircuitDecodeError(f"invalid type for {where}: expected a map")
    return {k: _decode_register(r, f"{where}[{k!r}]") for k, r in v.items()}


def _where(where, name: str | None = None) -> str:
    w = where() if callable(where) else where
    return w if name is None else f"{w}.{name}"


def decode_instruction(v: Any, where: Any = "instruction") -> Instruction:
    """``where``: the instruction's path for error messages (a string, or a
    callable producing it: formatted only when an error is raised)."""
    if not isinstance(v, dict):
        raise CircuitDecodeError(f"invalid type for {_where(where)}: expected internally tagged enum")
    if "kind" not in v:
        raise CircuitDecodeError(f"missing field `kind` in {_where(where)}")
    kind = v["kind"]
    if not isinstance(kind, str) or kind not in _FIELDS:
        raise CircuitDecodeError(f"unknown variant `{kind}` in {_where(where)}")
    out: dict[str, Any] = {}
    cond = None
    op = None
    for name, typ in _FIELDS[kind]:
        if name not in v:
            raise CircuitDecodeError(f"missing field `{name}` in {_where(where)} ({kind})")
        val = v[name]
        tv = type(val)
        if typ == "u":
            # fast path: a plain int in range (bool is not int here: type() is exact)
            out[name] = val if tv is int and 0 <= val <= _U64_MAX else _usize(val, _where(where, name))
        elif typ == "f":
            out[name] = val if tv is float and math.isfinite(val) else _f64(val, _where(where, name))
        elif typ == "s":
            out[name] = val if tv is str else _string(val, _where(where, name))
        elif typ == "fl":
            if not isinstance(val, list):
                raise CircuitDecodeError(f"invalid type for {_where(where, name)}: expected a sequence")
            out[name] = [_f64(x, _where(where, name)) for x in val]
        elif typ == "ul":
            if not isinstance(val, list):
                raise CircuitDecodeError(f"invalid type for {_where(where, name)}: expected a sequence")
            out[name] = [_usize(x, _where(where, name)) for x in val]
        elif typ == "cond":
            w = _where(where, name)
            if not isinstance(val, dict):
                raise CircuitDecodeError(f"invalid type for {w}: expected struct Condition")
            for f in ("creg_base", "creg_size", "creg_value"):
                if f not in val:
                    raise CircuitDecodeError(f"missing field `{f}` in {w}")
            cond = (_usize(val["creg_base"], w), _usize(val["creg_size"], w),
                    _usize(val["creg_value"], w))
        elif typ == "inst":
            op = decode_instruction(val, _where(where, name))
    return Instruction(kind, out, cond, op)


def decode_circuit_obj(obj: Any) -> Circuit:
    if not isinstance(obj, dict):
        raise CircuitDecodeError("invalid type: expected struct Circuit")
    if "qregs" not in obj:
        raise CircuitDecodeError("missing field `qregs`")
    if "instructions" not in obj:
        raise CircuitDecodeError("missing field `instructions`")
    qregs = _decode_registers(obj["qregs"], "qregs")
    cregs = _decode_registers(obj["cregs"], "cregs") if "cregs" in obj else {}
    insts = obj["instructions"]
    if not isinstance(insts, list):
        raise CircuitDecodeError("invalid type for instructions: expected a sequence")
    return Circuit(qregs, cregs, [decode_instruction(x, lambda i=i: f"instructions[{i}]")
                                  for i, x in enumerate(insts)])


def _reject_constant(c: str):
    raise CircuitDecodeError(f"invalid JSON number {c}")


def decode_circuit_json(text: str) -> Circuit:
    """Decode ``model_dump_json()`` output (serde_json semantics)."""
    try:
        obj = json.loads(text, parse_constant=_reject_constant)
    except CircuitDecodeError:
        raise
    except (ValueError, TypeError) as e:
        raise CircuitDecodeError(str(e)) from None
    return decode_circuit_obj(obj)


# ---- encoding to dq_inst ------------------------------------------------------------


@dataclass
class Program:
    """A circuit encoded for ``dq_run``."""

    insts: np.ndarray          # INST_DTYPE records
    conds: np.ndarray          # COND_DTYPE records
    num_qubits: int
    num_cbits: int             # formatted width (max creg base+size)
    cbit_space: int            # length of the cbits array (covers every cbit used)
    gate_names: dict[int, str]  # instruction index -> generic gate name (lower-cased)

    @property
    def ninst(self) -> int:
        return int(self.insts.shape[0])


_NEG8 = (-1,) * MAX_INST_QUBITS
_ZERO4 = (0.0, 0.0, 0.0, 0.0)
_TWO_QUBIT_GENERIC = {KIND["g_phi_plus"], KIND["g_psi_minus"], KIND["g_psi_plus"], KIND["g_cz"],
                      KIND["g_cx"]}
# per kind: (dq kind, qubit field names, parameter field names)
_SPEC = {
    k: (KIND[k] if k in KIND else -1, tuple(n for n, t in v if t == "u" and n != "cbit"),
        tuple(n for n, t in v if t == "f"))
    for k, v in _FIELDS.items()
}


def _encode_one(inst: Instruction, conds: list[tuple[int, int, int]], names: dict, idx: int,
                chain: list[tuple[int, int, int]]) -> tuple[tuple, int]:
    """(dq_inst record as a tuple, highest cbit index referenced or -1)."""
    if inst.kind == "conditional":
        return _encode_one(inst.op, conds, names, idx, chain + [inst.condition])
    max_cbit = -1
    f = inst.fields
    cbit = 0
    q = _NEG8
    p = _ZERO4
    if inst.kind == "gate":
        lname = f["name"].lower()
        if lname in _GENERIC:
            kind = KIND[_GENERIC[lname]]
        elif lname.startswith("circuit-"):
            kind = KIND["g_opaque"]
        else:
            kind = KIND["g_unsupported"]
        names[idx] = lname
        qs = f["qubits"]
        nq = min(len(qs), MAX_INST_QUBITS)
        if kind in _TWO_QUBIT_GENERIC:
            if len(qs) != 2:
                raise ValueError(f"generic gate {f['name']!r} expects 2 qubits, got {len(qs)}")
            nq = 2
        ql = [qv if qv < (1 << 31) else -1 for qv in qs[:MAX_INST_QUBITS]]
        q = tuple(ql) + _NEG8[len(ql):]
    elif inst.kind in ("barrier", "classical"):
        kind = KIND[inst.kind]
        nq = 0
    else:
        kind, qn, pn = _SPEC[inst.kind]
        nq = len(qn)
        ql = []
        for n in qn:
            v = f[n]
            if v >= (1 << 31):
                raise ValueError(f"qubit index {v} out of range")
            ql.append(v)
        q = tuple(ql) + _NEG8[nq:]
        if pn:
            pl = [f[n] for n in pn]
            p = tuple(pl) + _ZERO4[len(pl):]
        if inst.kind == "measure":
            cbit = f["cbit"]
            max_cbit = cbit
    cond_first = cond_count = 0
    if chain:
        cond_first = len(conds)
        cond_count = len(chain)
        for c in chain:
            if c[1] > 64:
                raise ValueError("conditions wider than 64 classical bits are not supported")
            conds.append(c)
            if c[1] > 0:
                max_cbit = max(max_cbit, c[0] + c[1] - 1)
    return (kind, nq, q, cbit, p, cond_first, cond_count), max_cbit


def encode(circuit: Circuit) -> Program:
    n = circuit.num_qubits()
    conds: list[tuple[int, int, int]] = []
    names: dict[int, str] = {}
    max_cbit = -1
    rows = []
    for i, inst in enumerate(circuit.instructions):
        row, mc = _encode_one(inst, conds, names, i, [])
        rows.append(row)
        if mc > max_cbit:
            max_cbit = mc
    insts = np.array(rows, dtype=INST_DTYPE) if rows else np.zeros(0, dtype=INST_DTYPE)
    carr = np.zeros(len(conds), dtype=COND_DTYPE)
    for i, (b, s_, v) in enumerate(conds):
        carr[i] = (b, s_, v)
    ncb = circuit.num_cbits()
    space = max(ncb, max_cbit + 1, 1)
    if space > (1 << 26):
        raise ValueError("classical register index too large")
    return Program(insts, carr, n, ncb, space, names)


def _decode_native(text: str) -> Program | None:
    """The library's decoder (``dq_circuit_decode``); None when it leaves the
    text to :func:`decode_circuit_json` (an error to report, or a rare form)."""
    from . import _native as nat

    try:
        raw = text.encode("utf-8")
    except UnicodeEncodeError:  # lone surrogates in the text
        return None
    L = nat.lib()
    handle = ctypes.c_void_p()
    info = nat.CircuitInfo()
    rc = L.dq_circuit_decode(raw, len(raw), ctypes.byref(handle), ctypes.byref(info))
    if rc == nat.DQ_ERR_DECODE:
        return None
    nat.check(rc, "dq_circuit_decode")
    try:
        insts = np.empty(info.ninst, dtype=INST_DTYPE)
        conds = np.empty(info.ncond, dtype=COND_DTYPE)
        names = np.empty(info.names_bytes, dtype=np.uint8)
        nat.check(L.dq_circuit_export(handle, nat.ptr(insts) if insts.size else None,
                                      nat.ptr(conds) if conds.size else None,
                                      nat.ptr(names) if names.size else None),
                  "dq_circuit_export")
    finally:
        L.dq_circuit_free(handle)
    gate_names: dict[int, str] = {}
    buf = names.tobytes()
    pos = 0
    while pos < len(buf):
        idx, ln = struct.unpack_from("<QQ", buf, pos)
        gate_names[idx] = buf[pos + 16:pos + 16 + ln].decode("utf-8")
        pos += 16 + ln
    return Program(insts, conds, int(info.num_qubits), int(info.num_cbits), int(info.cbit_space),
                   gate_names)


def decode_program(text: str) -> Program:
    """Circuit JSON -> ``Program``: the library's decoder for the well-formed
    case, this module's decoder and encoder for everything it declines (same
    result, and the reference's error messages)."""
    prog = _decode_native(text)
    if prog is not None:
        return prog
    return encode(decode_circuit_json(text))


def circuit_json(circuit: Any) -> str:
    """The reference's boundary call: ``circuit.model_dump_json()`` (simulator.rs:327-329)."""
    s = circuit.model_dump_json()
    if not isinstance(s, str):
        raise TypeError(f"model_dump_json() returned {type(s).__name__}, expected str")
    return s


def format_cbits(bits: np.ndarray, num_cbits: int) -> str:
    """``format_cbits`` (src/types.rs:43-51): MSB first, unwritten bits read 0."""
    if num_cbits == 0:
        return ""
    return "".join("1" if bits[i] > 0 else "0" for i in range(num_cbits - 1, -1, -1))
