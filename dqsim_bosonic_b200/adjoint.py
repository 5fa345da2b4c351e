"""Expectation values of Pauli sums and their adjoint gradients.

The reference engine has no gradients; this module adds differentiation of
``<psi(theta)|H|psi(theta)>`` on top of the same statevector engine:

* :class:`PauliSum` — an observable ``H = sum_t c_t P_t`` (real ``c_t``).
* :class:`ParamCircuit` — a unitary gate list whose angles are fixed numbers
  or trainable :class:`Param` references into a parameter vector ``theta``.
* :func:`adjoint_gradient` — ``E`` and ``dE/dtheta`` in one forward and one
  reverse sweep (``dq_adjoint``: uncompute-by-inverse-gates, no stored
  intermediate states).
* :func:`parameter_shift_gradient` — the shift-rule baseline, 2 or 4 forward
  runs per differentiated gate parameter.
* :func:`expval` — a ``torch.autograd.Function`` front end: the forward runs
  the adjoint pass and keeps the gradient for backward.

All device work goes through ``libdqsim_cuda.so``; nothing here computes
amplitudes on the host.
"""
from __future__ import annotations

import ctypes
import math
import re
import threading
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _native as nat

__all__ = [
    "PauliSum",
    "Param",
    "ParamCircuit",
    "expectation",
    "adjoint_gradient",
    "adjoint_gradient_batch",
    "parameter_shift_gradient",
    "AdjointExpectation",
    "expval",
    "DIFFERENTIABLE_KINDS",
]

# angle parameters per kind (dq_adjoint differentiates these)
DIFFERENTIABLE_KINDS = {
    "rx": 1, "ry": 1, "rz": 1, "p": 1, "u1": 1, "u2": 2, "u3": 3, "u": 3,
    "crx": 1, "cry": 1, "crz": 1, "cp": 1, "cu1": 1, "cu3": 3, "cu": 4,
    "rxx": 1, "rzz": 1,
}
# parameters every gate kind takes (fixed or trainable)
_PARAM_COUNT = dict(DIFFERENTIABLE_KINDS)
_QUBITS = {
    **{k: 1 for k in ("id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "u0",
                      "rx", "ry", "rz", "p", "u1", "u2", "u3", "u")},
    **{k: 2 for k in ("cx", "cz", "cy", "ch", "swap", "csx", "crx", "cry", "crz", "cu1", "cp",
                      "cu3", "cu", "rxx", "rzz")},
    **{k: 3 for k in ("ccx", "cswap", "rccx")},
    **{k: 4 for k in ("rc3x", "c3x", "c3sqrtx")},
    "c4x": 5,
}


# ---- observables ------------------------------------------------------------------------

_TOKEN = re.compile(r"^([IXYZ])(\d+)$")


class PauliSum:
    """``H = sum_t coeff_t * P_t`` with ``P_t`` a tensor product of Paulis.

    A term is ``(coeff, spec)`` where ``spec`` is a string of tokens such as
    ``"Z0 Z1"`` / ``"X3"`` / ``"Y0 Z2"`` (``""`` or ``"I"`` is the identity),
    or a dict ``{qubit: "X" | "Y" | "Z"}``.  Qubit ``q`` is bit ``q`` of the
    state index, as everywhere in the engine.
    """

    def __init__(self, terms=()):
        self._c: list[float] = []
        self._x: list[int] = []
        self._z: list[int] = []
        for coeff, spec in terms:
            self.add(coeff, spec)

    def add(self, coeff: float, spec) -> "PauliSum":
        c = float(coeff)
        if not math.isfinite(c):
            raise ValueError("Pauli coefficient must be finite")
        ops = {}
        if isinstance(spec, dict):
            items = spec.items()
        else:
            items = []
            for tok in str(spec).split():
                if tok == "I":
                    continue
                m = _TOKEN.match(tok)
                if not m:
                    raise ValueError(f"bad Pauli token {tok!r} (expected e.g. 'X0', 'Z12')")
                items.append((int(m.group(2)), m.group(1)))
        x = z = 0
        for q, op in items:
            q = int(q)
            op = str(op).upper()
            if q < 0 or q >= 64:
                raise ValueError(f"qubit {q} out of range")
            if q in ops:
                raise ValueError(f"qubit {q} appears twice in one Pauli term")
            ops[q] = op
            if op == "I":
                continue
            if op not in ("X", "Y", "Z"):
                raise ValueError(f"bad Pauli operator {op!r}")
            if op in ("X", "Y"):
                x |= 1 << q
            if op in ("Z", "Y"):
                z |= 1 << q
        self._c.append(c)
        self._x.append(x)
        self._z.append(z)
        return self

    def __len__(self) -> int:
        return len(self._c)

    @property
    def num_qubits(self) -> int:
        m = 0
        for x, z in zip(self._x, self._z):
            m = max(m, (x | z).bit_length())
        return m

    def array(self) -> np.ndarray:
        """The terms as a ``dq_pauli_term`` record array."""
        a = np.zeros(len(self._c), dtype=nat.PAULI_DTYPE)
        a["coeff"] = self._c
        a["xmask"] = np.array(self._x, dtype=np.uint64)
        a["zmask"] = np.array(self._z, dtype=np.uint64)
        return a


# ---- parametrised circuits ------------------------------------------------------------------

@dataclass(frozen=True)
class Param:
    """Angle = ``scale * theta[index] + shift``."""

    index: int
    scale: float = 1.0
    shift: float = 0.0


class ParamCircuit:
    """A unitary gate list with fixed or trainable angles.

    ``add(kind, qubits, params)`` takes the engine's gate kinds (``"ry"``,
    ``"cx"``, ``"rzz"``, ...) with the reference's parameter order (``u3``:
    theta, phi, lam; ``cu``: theta, phi, lam, gamma; ``rz``/``p``/``cp``: one
    angle) and the reference's qubit order (controls first).  Every kind has a
    method of the same name, e.g. ``c.ry(0, Param(3))``, ``c.cx(0, 1)``.
    """

    def __init__(self, num_qubits: int, num_params: int | None = None):
        if num_qubits < 1 or num_qubits > 34:
            raise ValueError("num_qubits must be in 1..34")
        self.num_qubits = int(num_qubits)
        self._declared = num_params
        self.ops: list[tuple[str, tuple[int, ...], tuple]] = []

    @property
    def num_params(self) -> int:
        m = 0
        for _, _, ps in self.ops:
            for p in ps:
                if isinstance(p, Param):
                    m = max(m, p.index + 1)
        if self._declared is not None:
            if m > self._declared:
                raise ValueError("a Param index exceeds the declared num_params")
            return int(self._declared)
        return m

    def add(self, kind: str, qubits, params=()) -> "ParamCircuit":
        kind = str(kind).lower()
        if kind not in _QUBITS:
            raise ValueError(f"unsupported gate kind {kind!r} for a parametrised circuit")
        qs = tuple(int(q) for q in (qubits if isinstance(qubits, (list, tuple)) else [qubits]))
        if len(qs) != _QUBITS[kind]:
            raise ValueError(f"{kind} takes {_QUBITS[kind]} qubits, got {len(qs)}")
        if len(set(qs)) != len(qs):
            raise ValueError(f"repeated qubit in {kind}{qs}")
        for q in qs:
            if q < 0 or q >= self.num_qubits:
                raise ValueError(f"qubit {q} out of range for {self.num_qubits} qubits")
        ps = tuple(params)
        need = _PARAM_COUNT.get(kind, 0)
        if len(ps) != need:
            raise ValueError(f"{kind} takes {need} parameters, got {len(ps)}")
        for p in ps:
            if isinstance(p, Param):
                if p.index < 0:
                    raise ValueError("Param index must be >= 0")
            elif not math.isfinite(float(p)):
                raise ValueError("fixed angles must be finite")
        self.ops.append((kind, qs, ps))
        return self

    def __getattr__(self, kind):
        if kind.startswith("_") or kind not in _QUBITS:
            raise AttributeError(kind)
        nq = _QUBITS[kind]

        def method(*args):
            return self.add(kind, args[:nq], args[nq:])

        return method

    def occurrences(self) -> list[tuple[int, int, Param]]:
        """(instruction, slot, Param) for every trainable angle, in program order."""
        out = []
        for i, (_, _, ps) in enumerate(self.ops):
            for j, p in enumerate(ps):
                if isinstance(p, Param):
                    out.append((i, j, p))
        return out

    def bind(self, theta) -> np.ndarray:
        """The program with every angle evaluated at ``theta`` (dq_inst records)."""
        th = np.asarray(theta, dtype=np.float64).reshape(-1)
        if th.size != self.num_params:
            raise ValueError(f"theta has {th.size} entries, the circuit {self.num_params}")
        insts = np.zeros(len(self.ops), dtype=nat.INST_DTYPE)
        insts["cbit"] = -1
        for i, (kind, qs, ps) in enumerate(self.ops):
            insts[i]["kind"] = nat.KIND[kind]
            insts[i]["nq"] = len(qs)
            insts[i]["q"][: len(qs)] = qs
            for j, p in enumerate(ps):
                insts[i]["p"][j] = (p.scale * th[p.index] + p.shift) if isinstance(p, Param) else float(p)
        return insts

    def param_slots(self) -> np.ndarray:
        """param_index for dq_adjoint: one gradient entry per trainable occurrence."""
        idx = np.full((len(self.ops), 4), -1, dtype=np.int32)
        for o, (i, j, _) in enumerate(self.occurrences()):
            idx[i, j] = o
        return idx


# ---- engine calls ------------------------------------------------------------------------------

_states: dict[tuple[int, int, int], nat.State] = {}
_states_lock = threading.Lock()


def _state(n: int, device: int, slot: int = 0) -> nat.State:
    """A cached engine state per (qubits, device, worker slot)."""
    key = (n, device, slot)
    with _states_lock:
        st = _states.get(key)
        if st is None:
            st = nat.State(n, device)
            _states[key] = st
        return st


def _exec_mode(exec: str) -> int:
    if exec == "fused":
        return nat.EXEC_FUSED
    if exec == "per_gate":
        return nat.EXEC_PER_GATE
    raise ValueError("exec must be 'fused' or 'per_gate'")


def _check_observable(circuit: ParamCircuit, observable: PauliSum) -> np.ndarray:
    if observable.num_qubits > circuit.num_qubits:
        raise ValueError("the observable acts on qubits outside the circuit")
    return observable.array()


def expectation(circuit: ParamCircuit, theta, observable: PauliSum, *, device: int = 0,
                exec: str = "fused") -> float:
    """``<0|U(theta)^dagger H U(theta)|0>`` by one forward run."""
    terms = _check_observable(circuit, observable)
    insts = circuit.bind(theta)
    return _forward_expval(circuit.num_qubits, insts, terms, device, _exec_mode(exec))


def _forward_expval(n, insts, terms, device, mode) -> float:
    L = nat.lib()
    st = _state(n, device)
    st.reset()
    opts = nat.RunOpts(nat.SEM_SIMULATE, mode, 0, 0, 0, 0)
    nat.check(L.dq_run(st.handle, nat.ptr(insts), len(insts), None, 0, 0, None, 0,
                       ctypes.byref(opts), None), "dq_run")
    out = ctypes.c_double(0.0)
    nat.check(L.dq_expval_pauli(st.handle, nat.ptr(terms), len(terms), ctypes.byref(out)),
              "dq_expval_pauli")
    return out.value


def adjoint_gradient(circuit: ParamCircuit, theta, observable: PauliSum, *, device: int = 0,
                     exec: str = "fused", timing: dict | None = None,
                     _slot: int = 0) -> tuple[float, np.ndarray]:
    """``(E, dE/dtheta)`` from one forward and one adjoint (reverse) pass.

    ``timing``: a dict that receives the device milliseconds of the forward
    pass, of lambda = H psi and of the backward pass, and the number of fused
    backward sweeps."""
    terms = _check_observable(circuit, observable)
    th = np.asarray(theta, dtype=np.float64).reshape(-1)
    insts = circuit.bind(th)
    occ = circuit.occurrences()
    slots = circuit.param_slots()
    st = _state(circuit.num_qubits, device, _slot)
    st.reset()
    opts = nat.RunOpts(nat.SEM_SIMULATE, _exec_mode(exec), 0, 0, 0, 0)
    e = ctypes.c_double(0.0)
    g_occ = np.zeros(max(1, len(occ)), dtype=np.float64)
    phases = np.zeros(4, dtype=np.float64)
    nat.check(nat.lib().dq_adjoint(st.handle, nat.ptr(insts), len(insts), nat.ptr(slots), len(occ),
                                   nat.ptr(terms), len(terms), ctypes.byref(opts), ctypes.byref(e),
                                   nat.ptr(g_occ), nat.ptr(phases) if timing is not None else None),
              "dq_adjoint")
    if timing is not None:
        timing.update(forward_ms=float(phases[0]), observable_ms=float(phases[1]),
                      backward_ms=float(phases[2]), backward_sweeps=int(phases[3]))
    grad = np.zeros(circuit.num_params, dtype=np.float64)
    for o, (_, _, p) in enumerate(occ):
        grad[p.index] += p.scale * g_occ[o]
    return e.value, grad


def adjoint_gradient_batch(circuit: ParamCircuit, thetas, observable: PauliSum, *,
                           device: int = 0, exec: str = "fused", workers: int = 0,
                           stats: dict | None = None):
    """``(E[B], dE/dtheta[B, P])`` for a batch of parameter sets.

    Default (``workers = 0``, fused exec): one ``dq_adjoint_batch`` call runs
    every set together -- each fused forward sweep, lambda = H psi and each
    fused backward sweep is ONE launch over all sets.  ``workers > 0``: the
    sets run one adjoint pass each, ``workers`` of them in flight at once on
    separate engine states (host threads).  ``stats``: a dict that receives
    the batched call's launch count, sweep counts and phase times."""
    th = np.asarray(thetas, dtype=np.float64)
    if th.ndim != 2:
        raise ValueError("thetas must be 2-D: (sets, parameters)")
    B = th.shape[0]
    if th.shape[1] != circuit.num_params:
        raise ValueError(f"thetas have {th.shape[1]} columns, the circuit {circuit.num_params}")
    es = np.empty(B)
    gs = np.empty((B, circuit.num_params))
    if workers <= 0 and _exec_mode(exec) == nat.EXEC_FUSED:
        return _adjoint_batch_native(circuit, th, observable, device, stats)
    workers = max(1, min(int(workers) if workers > 0 else 4, B))

    def run(w):
        for b in range(w, B, workers):
            es[b], gs[b] = adjoint_gradient(circuit, th[b], observable, device=device, exec=exec,
                                            _slot=w)

    if workers == 1:
        run(0)
    else:
        with ThreadPoolExecutor(max_workers=workers) as ex:
            for f in [ex.submit(run, w) for w in range(workers)]:
                f.result()
    return es, gs


def _adjoint_batch_native(circuit: ParamCircuit, th: np.ndarray, observable: PauliSum, device: int,
                          stats: dict | None):
    terms = _check_observable(circuit, observable)
    B = th.shape[0]
    insts = circuit.bind(th[0])
    occ = circuit.occurrences()
    slots = circuit.param_slots()
    idx = np.array([p.index for (_, _, p) in occ], dtype=np.int64)
    scale = np.array([p.scale for (_, _, p) in occ], dtype=np.float64)
    shift = np.array([p.shift for (_, _, p) in occ], dtype=np.float64)
    # value of every trainable occurrence in every set
    vals = np.ascontiguousarray(th[:, idx] * scale + shift) if len(occ) else np.zeros((B, 1))
    es = np.zeros(B, dtype=np.float64)
    g_occ = np.zeros((B, max(1, len(occ))), dtype=np.float64)
    st = nat.AdjointBatchStats()
    nat.check(nat.lib().dq_adjoint_batch(int(device), circuit.num_qubits, nat.ptr(insts), len(insts),
                                         nat.ptr(slots), len(occ), nat.ptr(vals), B, nat.ptr(terms),
                                         len(terms), nat.ptr(es), nat.ptr(g_occ), ctypes.byref(st)),
              "dq_adjoint_batch")
    if stats is not None:
        stats.update({name: getattr(st, name) for name, _ in nat.AdjointBatchStats._fields_})
    gs = np.zeros((B, circuit.num_params), dtype=np.float64)
    if len(occ):
        np.add.at(gs.T, idx, (g_occ[:, :len(occ)] * scale).T)
    return es, gs


# shift rules: (coefficient, shift) pairs; df/dx = sum c * f(x + s)
_S2 = ((0.5, math.pi / 2), (-0.5, -math.pi / 2))
_D1 = (math.sqrt(2) + 1) / (4 * math.sqrt(2))
_D2 = (math.sqrt(2) - 1) / (4 * math.sqrt(2))
_S4 = ((_D1, math.pi / 2), (-_D1, -math.pi / 2), (-_D2, 3 * math.pi / 2), (_D2, -3 * math.pi / 2))


def _shift_rule(kind: str, slot: int):
    """Two-term rule for generators with eigenvalue gap 1 (Pauli rotations,
    phases, the u3 angles), four-term rule for controlled rotations (generator
    |1><1| (x) P/2: gaps 1/2 and 1)."""
    if kind in ("crx", "cry", "crz"):
        return _S4
    if kind in ("cu3", "cu") and slot == 0:
        return _S4
    if kind in DIFFERENTIABLE_KINDS:
        return _S2
    raise ValueError(f"no shift rule for {kind}")


def parameter_shift_gradient(circuit: ParamCircuit, theta, observable: PauliSum, *,
                             device: int = 0, exec: str = "per_gate",
                             occurrences=None) -> np.ndarray:
    """dE/dtheta by the parameter-shift rule: each trainable occurrence is
    shifted on its own (2 or 4 forward runs), contributions summed per theta
    entry.  ``occurrences`` limits the work to a subset (indices into
    :meth:`ParamCircuit.occurrences`); the other entries get no contribution."""
    terms = _check_observable(circuit, observable)
    th = np.asarray(theta, dtype=np.float64).reshape(-1)
    base = circuit.bind(th)
    mode = _exec_mode(exec)
    occ = circuit.occurrences()
    sel = range(len(occ)) if occurrences is None else occurrences
    grad = np.zeros(circuit.num_params, dtype=np.float64)
    for o in sel:
        i, j, p = occ[o]
        kind = circuit.ops[i][0]
        g = 0.0
        for c, s in _shift_rule(kind, j):
            insts = base.copy()
            insts[i]["p"][j] += s
            g += c * _forward_expval(circuit.num_qubits, insts, terms, device, mode)
        grad[p.index] += p.scale * g
    return grad


# ---- torch front end ------------------------------------------------------------------------------

def _torch():
    import torch

    return torch


class AdjointExpectation:
    """``torch.autograd.Function``: ``E = expval(theta)`` with the adjoint
    gradient computed in the forward pass and applied in backward.  ``theta``
    is 1-D (one parameter set) or 2-D (a batch of parameter sets; ``E`` is
    then 1-D)."""

    _fn = None

    @classmethod
    def function(cls):
        if cls._fn is None:
            torch = _torch()

            class _Fn(torch.autograd.Function):
                @staticmethod
                def forward(ctx, theta, circuit, observable, device, exec, workers):
                    th = theta.detach().to("cpu", torch.float64).numpy()
                    batched = th.ndim == 2
                    rows = th if batched else th[None, :]
                    es, gs = adjoint_gradient_batch(circuit, rows, observable, device=device,
                                                    exec=exec, workers=workers)
                    grad = torch.from_numpy(gs if batched else gs[0]).to(theta.device, theta.dtype)
                    ctx.save_for_backward(grad)
                    ctx.batched = batched
                    e = torch.from_numpy(es if batched else es[:1].reshape(())).to(theta.device,
                                                                                  theta.dtype)
                    return e

                @staticmethod
                def backward(ctx, grad_out):
                    (grad,) = ctx.saved_tensors
                    g = grad_out.unsqueeze(-1) * grad if ctx.batched else grad_out * grad
                    return g, None, None, None, None, None

            cls._fn = _Fn
        return cls._fn


def expval(theta, circuit: ParamCircuit, observable: PauliSum, *, device: int = 0,
           exec: str = "fused", workers: int = 0):
    """Differentiable ``<H>`` (torch tensor in, torch tensor out); a 2-D
    ``theta`` is a batch of parameter sets, run together by one batched
    adjoint call (``workers > 0``: that many sets at a time on host threads)."""
    return AdjointExpectation.function().apply(theta, circuit, observable, device, exec, workers)
