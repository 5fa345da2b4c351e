"""mps.py — CPU restatement of the reference's MPS simulator (numpy).

TEST INFRASTRUCTURE ONLY.  This module is the parity oracle and the timed CPU
baseline of the MPS backend.  Only tests/, __graft_entry__.smoke() and
bench.py (its cpu_baseline leg) may import it, and only as the checker or the
baseline; the product path (dqsim_bosonic_b200) never imports it.

What it restates (src/monolithic/mps/simulator.rs of the dqsim crate):
  :36-63    Tensor: data[(left * 2 + state) * right + right_index]
  :79-96    Mps::new: every site |0>, bond dimension 1
  :98-113   apply_1q: new[l][o][r] = sum_i mat[o][i] old[l][i][r]
  :115-135  apply_2q: swap chain towards the low qubit, gate (reversed when
            a > b, reverse_2q_order :561-579), swap chain back
  :137-236  apply_adjacent_2q: theta[(l*2+o0), (o1*R+r)], thin SVD, keep =
            #(s > threshold) clamped to [1, max_bond], truncation_scale =
            total_norm / max(kept_norm, 1e-15) when discarded_weight > 0,
            left = U[:, :keep], right = (s * scale) Vt[:keep, :]
  :238-257  to_statevector: amplitude of basis i = product of the site
            matrices selected by the bits of i (qubit 0 first)
  :259-291  measure / project_qubit: p1 from the statevector (ascending
            index), clamp to [0, 1], outcome = draw < p1, scale by
            1 / sqrt(prob) (0 when prob = 0)
  :457-559  run_instruction: which instructions are gates, no-ops, errors
The SVD is LAPACK's (numpy.linalg.svd), not nalgebra 0.33's Golub-Kahan: the
singular vectors differ by a gauge, which every observable (statevector,
probabilities, outcomes) is invariant to, so parity is held to a tolerance.
The gate matrices and the ChaCha8 draws are injected by the caller (the C
oracle's restatements of gates.rs and rand_chacha).
"""
from __future__ import annotations

from typing import Callable

import numpy as np

# dq_kind values of the instruction records this oracle interprets
# (include/dqsim_cuda.h), passed in by the caller as a dict.


class Mps:
    def __init__(self, n: int, max_bond: int | None, threshold: float):
        self.n = n
        self.max_bond = max_bond
        self.threshold = threshold
        self.tensors = []
        for _ in range(n):
            t = np.zeros((1, 2, 1), dtype=np.complex128)
            t[0, 0, 0] = 1.0
            self.tensors.append(t)
        self.svd_calls = 0

    def bond_dims(self) -> list[int]:
        return [1] + [t.shape[2] for t in self.tensors]

    def apply_1q(self, q: int, m: np.ndarray) -> None:
        old = self.tensors[q]
        new = np.empty_like(old)
        new[:, 0, :] = m[0, 0] * old[:, 0, :] + m[0, 1] * old[:, 1, :]
        new[:, 1, :] = m[1, 0] * old[:, 0, :] + m[1, 1] * old[:, 1, :]
        self.tensors[q] = new

    def apply_2q(self, a: int, b: int, m: np.ndarray, swap: np.ndarray) -> None:
        if a == b:
            return
        lo, hi, rev = (a, b, False) if a < b else (b, a, True)
        for pos in range(hi - 1, lo, -1):
            self.apply_adjacent_2q(pos, swap)
        self.apply_adjacent_2q(lo, reverse_2q_order(m) if rev else m)
        for pos in range(lo + 1, hi):
            self.apply_adjacent_2q(pos, swap)

    def apply_adjacent_2q(self, q: int, m: np.ndarray) -> None:
        A, B = self.tensors[q], self.tensors[q + 1]
        L, R = A.shape[0], B.shape[2]
        # inp[l, i0, i1, r] = sum_k A[l, i0, k] B[k, i1, r]
        inp = np.einsum("aik,kjb->aijb", A, B)
        g = m.reshape(2, 2, 2, 2)  # [o0, o1, i0, i1]
        out = np.einsum("xyij,aijb->axyb", g, inp)  # [l, o0, o1, r]
        theta = out.reshape(L * 2, 2 * R)  # row = l*2+o0, col = o1*R + r
        u, s, vt = np.linalg.svd(theta, full_matrices=False)
        self.svd_calls += 1
        keep = max(int(np.count_nonzero(s > self.threshold)), 1)
        if self.max_bond is not None:
            keep = min(keep, max(self.max_bond, 1))
        kept_norm = max(float(np.sqrt(np.sum(s[:keep] ** 2))), 1e-15)
        total_norm = float(np.sqrt(np.sum(s ** 2)))
        discarded = float(np.sum(s[keep:] ** 2))
        scale = total_norm / kept_norm if discarded > 0.0 else 1.0
        self.tensors[q] = u[:, :keep].reshape(L, 2, keep).copy()
        self.tensors[q + 1] = ((s[:keep] * scale)[:, None] * vt[:keep, :]).reshape(keep, 2, R).copy()

    def to_statevector(self) -> np.ndarray:
        work = np.ones((1, 1), dtype=np.complex128)  # rows: basis bits of qubits < k
        for k, t in enumerate(self.tensors):
            w0 = work @ t[:, 0, :]
            w1 = work @ t[:, 1, :]
            work = np.concatenate([w0, w1], axis=0)  # bit k of the row index = state
        return work[:, 0].copy()

    def measure(self, q: int, draw: Callable[[], float]) -> int:
        st = self.to_statevector()
        idx = np.arange(st.size)
        sel = st[((idx >> q) & 1) == 1]
        p1 = 0.0
        for a in sel:  # ascending index, sequential sum
            p1 += a.real * a.real + a.imag * a.imag
        p1 = min(max(p1, 0.0), 1.0)
        outcome = 1 if draw() < p1 else 0
        prob = p1 if outcome == 1 else 1.0 - p1
        scale = 1.0 / np.sqrt(prob) if prob > 0.0 else 0.0
        t = self.tensors[q]
        t[:, outcome, :] = t[:, outcome, :] * scale
        t[:, 1 - outcome, :] = 0.0
        return outcome


def reverse_2q_order(m: np.ndarray) -> np.ndarray:
    """reverse_2q_order (simulator.rs:561-579): the gate with its qubits exchanged."""
    out = np.empty((4, 4), dtype=np.complex128)
    for a0 in range(2):
        for b0 in range(2):
            for a1 in range(2):
                for b1 in range(2):
                    out[a0 * 2 + b0, a1 * 2 + b1] = m[b0 * 2 + a0, b1 * 2 + a1]
    return out


class Unsupported(Exception):
    """An instruction the MPS dispatcher rejects (simulator.rs:540-557)."""

    def __init__(self, index: int):
        super().__init__(index)
        self.index = index


def run(insts: np.ndarray, conds: np.ndarray, n: int, ncbits: int, draw: Callable[[], float],
        matrix: Callable[[dict], tuple[str, np.ndarray | None]], max_bond: int | None = None,
        threshold: float = 1e-12) -> tuple[Mps, np.ndarray]:
    """MpsSimulator::simulate's instruction loop over encoded instruction records.

    ``matrix(inst)`` classifies one record: ("noop", None), ("1q", 2x2),
    ("2q", 4x4), ("measure", None), ("reset", None) or ("fail", None).
    Returns the MPS and the cbit array (-1 = never written).
    """
    mps = Mps(n, max_bond, threshold)
    cbits = np.full(max(ncbits, 1), -1, dtype=np.int64)
    swap = np.eye(4, dtype=np.complex128)[[0, 2, 1, 3]]
    xm = np.array([[0, 1], [1, 0]], dtype=np.complex128)
    for i, rec in enumerate(insts):
        ok = True
        for c in range(int(rec["cond_count"])):
            cd = conds[int(rec["cond_first"]) + c]
            actual = 0
            for bit in range(int(cd["creg_size"])):
                j = int(cd["creg_base"]) + bit
                v = int(cbits[j]) if j < cbits.size and cbits[j] > 0 else 0
                actual |= v << bit
            if actual != int(cd["creg_value"]):
                ok = False
                break
        if not ok:
            continue
        what, m = matrix(rec)
        q = [int(x) for x in rec["q"][: int(rec["nq"])]]
        if what == "noop":
            continue
        if what == "1q":
            mps.apply_1q(q[0], m)
        elif what == "2q":
            mps.apply_2q(q[0], q[1], m, swap)
        elif what == "measure":
            cbits[int(rec["cbit"])] = mps.measure(q[0], draw)
        elif what == "reset":
            if mps.measure(q[0], draw) == 1:
                mps.apply_1q(q[0], xm)
        else:
            raise Unsupported(i)
    return mps, cbits
