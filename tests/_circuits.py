"""Circuit builders for the tests and the benchmark.

A circuit is any object with ``model_dump_json()`` (the reference's only
requirement, statevector/simulator.rs:327-329).  ``JsonCircuit`` emits the
bosonic-model JSON layout the reference decodes (src/types.rs:8-135),
including the extra ``qubits``/``params`` keys that serde ignores.
"""
from __future__ import annotations

import json
import math

import numpy as np

_Q1 = ("qubit",)
_FIELDS = {
    "id": _Q1, "x": _Q1, "y": _Q1, "z": _Q1, "h": _Q1, "s": _Q1, "sdg": _Q1, "t": _Q1,
    "tdg": _Q1, "sx": _Q1, "sxdg": _Q1, "u0": _Q1, "reset": _Q1,
    "u3": ("qubit", "theta", "phi", "lam"), "u": ("qubit", "theta", "phi", "lam"),
    "u2": ("qubit", "phi", "lam"), "u1": ("qubit", "lam"), "p": ("qubit", "lam"),
    "rx": ("qubit", "theta"), "ry": ("qubit", "theta"), "rz": ("qubit", "phi"),
    "cx": ("control", "target"), "cz": ("control", "target"), "cy": ("control", "target"),
    "ch": ("control", "target"), "csx": ("control", "target"), "swap": ("a", "b"),
    "crx": ("control", "target", "theta"), "cry": ("control", "target", "theta"),
    "crz": ("control", "target", "lam"), "cu1": ("control", "target", "lam"),
    "cp": ("control", "target", "lam"), "cu3": ("control", "target", "theta", "phi", "lam"),
    "cu": ("control", "target", "theta", "phi", "lam", "gamma"),
    "rxx": ("a", "b", "theta"), "rzz": ("a", "b", "theta"),
    "ccx": ("control1", "control2", "target"), "rccx": ("control1", "control2", "target"),
    "cswap": ("control", "target1", "target2"),
    "rc3x": ("control1", "control2", "control3", "target"),
    "c3x": ("control1", "control2", "control3", "target"),
    "c3sqrtx": ("control1", "control2", "control3", "target"),
    "c4x": ("control1", "control2", "control3", "control4", "target"),
    "measure": ("qubit", "cbit"),
}
QUBIT_FIELDS = {"qubit", "control", "target", "a", "b", "control1", "control2", "control3",
                "control4", "target1", "target2"}
GATE_ARITY = {k: sum(1 for f in v if f in QUBIT_FIELDS) for k, v in _FIELDS.items()}
GATE_NPARAMS = {k: sum(1 for f in v if f not in QUBIT_FIELDS and f != "cbit") for k, v in _FIELDS.items()}
UNITARY_KINDS = [k for k in _FIELDS if k not in ("measure", "reset")]


def g(kind: str, *args) -> dict:
    """Instruction dict from positional field values in reference field order."""
    names = _FIELDS[kind]
    if len(args) != len(names):
        raise TypeError(f"{kind} takes {len(names)} values")
    d = {"kind": kind}
    d.update(dict(zip(names, args)))
    qs = [d[n] for n in names if n in QUBIT_FIELDS]
    d["qubits"] = qs   # bosonic-model extras, ignored by the decoder
    d["params"] = [d[n] for n in names if n not in QUBIT_FIELDS and n != "cbit"]
    return d


def gate(name: str, qubits, params=()) -> dict:
    return {"kind": "gate", "name": name, "params": list(params), "qubits": list(qubits)}


def cond(base: int, size: int, value: int, op: dict) -> dict:
    return {"kind": "conditional", "condition": {"creg_base": base, "creg_size": size,
                                                 "creg_value": value}, "op": op,
            "qubits": op.get("qubits", [])}


class JsonCircuit:
    def __init__(self, n: int, instructions: list, ncbits: int = 0, qregs=None, cregs=None):
        self.n = n
        self.instructions = list(instructions)
        self.qregs = qregs if qregs is not None else {"q": {"name": "q", "size": n, "base": 0}}
        if cregs is not None:
            self.cregs = cregs
        else:
            self.cregs = {"c": {"name": "c", "size": ncbits, "base": 0}} if ncbits else {}

    def to_dict(self) -> dict:
        return {"qregs": self.qregs, "cregs": self.cregs, "instructions": self.instructions}

    def model_dump_json(self) -> str:
        return json.dumps(self.to_dict())


def random_gate(rng: np.random.Generator, n: int, kind: str | None = None) -> dict:
    kinds = [k for k in UNITARY_KINDS if GATE_ARITY[k] <= n and k != "u0"]
    kind = kind or kinds[rng.integers(len(kinds))]
    qs = rng.choice(n, size=GATE_ARITY[kind], replace=False).tolist()
    ps = (rng.uniform(0, 2 * math.pi, size=GATE_NPARAMS[kind])).tolist()
    vals = []
    qi = pi = 0
    for f in _FIELDS[kind]:
        if f in QUBIT_FIELDS:
            vals.append(qs[qi]); qi += 1
        else:
            vals.append(ps[pi]); pi += 1
    return g(kind, *vals)


def random_circuit(seed: int, n: int, depth: int) -> JsonCircuit:
    rng = np.random.default_rng(seed)
    return JsonCircuit(n, [random_gate(rng, n) for _ in range(depth)])


# ---- the benchmark workloads --------------------------------------------------------------


def brickwork_u3_cx(n: int = 20, layers: int = 20, seed: int = 1234) -> JsonCircuit:
    """u3 on every qubit (angles ~ U[0, 2pi), seeded) then cx on brickwork pairs."""
    rng = np.random.default_rng(seed)
    insts = []
    for layer in range(layers):
        ang = rng.uniform(0.0, 2.0 * math.pi, size=(n, 3))
        for q in range(n):
            insts.append(g("u3", q, *ang[q].tolist()))
        start = 0 if layer % 2 == 0 else 1
        for q in range(start, n - 1, 2):
            insts.append(g("cx", q, q + 1))
    return JsonCircuit(n, insts)


def ragged_batch(count: int = 1024, seed: int = 99, n_lo: int = 10, n_hi: int = 22,
                 d_lo: int = 5, d_hi: int = 40) -> list:
    """Independent u3 + cx brickwork circuits of uneven size: n ~ U{n_lo..n_hi}
    qubits and depth ~ U{d_lo..d_hi} layers (each layer u3 on every qubit with
    angles ~ U[0, 2pi), then cx on the brickwork pairs), seeded."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(n_lo, n_hi + 1, size=count)
    ds = rng.integers(d_lo, d_hi + 1, size=count)
    return [brickwork_u3_cx(int(n), int(d), seed=int(seed) * 100003 + k)
            for k, (n, d) in enumerate(zip(ns, ds))]


def hadamard_diagonal_circuit(n, layers, seed):
    """Layers of Hadamards on random qubit subsets with random diagonal gates in between:
    register phases made only of Hadamards, whose pending phases pair them with qubits
    above and below them, local or not (the straight-line H phases of the sweep kernel)."""
    rng = np.random.default_rng(seed)
    insts = []
    diag2 = ["cp", "crz", "cu1", "rzz", "cz"]
    diag1 = ["p", "rz", "t", "s", "sdg", "z"]
    for _ in range(layers):
        for q in rng.permutation(n)[: int(rng.integers(1, n + 1))]:
            insts.append(g("h", int(q)))
        for _ in range(int(rng.integers(1, 2 * n))):
            if rng.random() < 0.6:
                a, b = (int(v) for v in rng.permutation(n)[:2])
                k = diag2[rng.integers(len(diag2))]
                insts.append(g(k, a, b) if k == "cz" else g(k, a, b, float(rng.uniform(-3, 3))))
            else:
                q = int(rng.integers(n))
                k = diag1[rng.integers(len(diag1))]
                insts.append(g(k, q, float(rng.uniform(-3, 3))) if k in ("p", "rz") else g(k, q))
    return JsonCircuit(n, insts)


def qft_with_x(n: int = 30, seed: int = 1234) -> JsonCircuit:
    """x on a seeded random subset (p = 0.5), then the textbook QFT with swaps."""
    rng = np.random.default_rng(seed)
    insts = [g("x", q) for q in range(n) if rng.random() < 0.5]
    for j in range(n):
        insts.append(g("h", j))
        for k in range(j + 1, n):
            insts.append(g("cp", k, j, math.pi / (2 ** (k - j))))
    for j in range(n // 2):
        insts.append(g("swap", j, n - 1 - j))
    return JsonCircuit(n, insts)


def distributed_qft_variant(n_data: int = 14, seed: int = 1234) -> JsonCircuit:
    """Two nodes of n_data data qubits plus one link qubit each, lowered to one
    register: node A data 0..n_data-1, link n_data; node B link n_data+1, data
    after it.  remote_link_psi_minus on the links, nonlocal_cz across data."""
    rng = np.random.default_rng(seed)
    n = 2 * n_data + 2
    la, lb = n_data, n_data + 1
    a_data = list(range(n_data))
    b_data = list(range(n_data + 2, n))
    insts = [g("h", q) for q in a_data + b_data]
    insts.append(gate("remote_link_psi_minus", [la, lb]))
    for i in range(n_data):
        insts.append(gate("nonlocal_cz", [a_data[i], b_data[(i + 3) % n_data]]))
        insts.append(g("rz", a_data[i], float(rng.uniform(-math.pi, math.pi))))
    insts.append(gate("remote_link_psi_minus", [la, lb]))
    for j in range(n):
        insts.append(g("h", j))
    return JsonCircuit(n, insts)


def trajectory_circuit(n: int = 16, layers: int = 12, seed: int = 7) -> JsonCircuit:
    """u3 + cx brickwork with measure q0 -> c0, conditional x q1 on c0 == 1 and
    reset q0 after every third layer."""
    rng = np.random.default_rng(seed)
    insts = []
    for layer in range(layers):
        ang = rng.uniform(0.0, 2.0 * math.pi, size=(n, 3))
        for q in range(n):
            insts.append(g("u3", q, *ang[q].tolist()))
        start = 0 if layer % 2 == 0 else 1
        for q in range(start, n - 1, 2):
            insts.append(g("cx", q, q + 1))
        if layer % 3 == 2:
            insts.append(g("measure", 0, 0))
            insts.append(cond(0, 1, 1, g("x", 1)))
            insts.append(g("reset", 0))
    return JsonCircuit(n, insts, ncbits=1)


def hea_ansatz(n: int, layers: int, seed: int):
    """ry then rz on every qubit, then rzz on the ring (i, i+1 mod n).
    Returns (circuit, parameter vector) with angles ~ U[-pi, pi)."""
    rng = np.random.default_rng(seed)
    params = rng.uniform(-math.pi, math.pi, size=layers * 3 * n)
    insts = []
    k = 0
    for _ in range(layers):
        for q in range(n):
            insts.append(g("ry", q, float(params[k]))); k += 1
        for q in range(n):
            insts.append(g("rz", q, float(params[k]))); k += 1
        for q in range(n):
            insts.append(g("rzz", q, (q + 1) % n, float(params[k]))); k += 1
    return JsonCircuit(n, insts), params


def hea_param_circuit(n: int, layers: int, seed: int, ham_seed: int = 5, ring: bool = True):
    """The hardware-efficient ansatz as a ParamCircuit: per layer ry then rz on
    every qubit, then rzz on the ring (i, i+1 mod n); angles ~ U[-pi, pi).
    H = sum_i a_i Z_i Z_{i+1} + sum_i b_i X_i, a, b ~ N(0, 1).
    Returns (circuit, theta, observable)."""
    from dqsim_bosonic_b200.adjoint import Param, ParamCircuit, PauliSum

    rng = np.random.default_rng(seed)
    theta = rng.uniform(-math.pi, math.pi, size=layers * 3 * n)
    c = ParamCircuit(n)
    k = 0
    pairs = [(q, (q + 1) % n) for q in range(n if ring else n - 1)]
    for _ in range(layers):
        for q in range(n):
            c.ry(q, Param(k)); k += 1
        for q in range(n):
            c.rz(q, Param(k)); k += 1
        for a, b in pairs:
            c.rzz(a, b, Param(k)); k += 1
    theta = theta[:k]
    hr = np.random.default_rng(ham_seed)
    a = hr.normal(size=len(pairs))
    b = hr.normal(size=n)
    H = PauliSum()
    for (i, j), ai in zip(pairs, a):
        H.add(float(ai), {i: "Z", j: "Z"})
    for i, bi in enumerate(b):
        H.add(float(bi), {i: "X"})
    return c, theta, H
