"""Writes the amplitude-level golden fixtures ``amp_*.json`` of this directory.

A probability cannot see a phase convention: rz(phi) and rz(-phi) give the
same distribution, and so do psi_minus and psi_plus on |00>.  These fixtures
pin the amplitudes themselves.  Each one is a small circuit in the
bosonic-model JSON layout the reference decodes (src/types.rs:8-135) and its
exact final statevector, written out below as closed-form expressions of
the gate definitions in src/gates.rs (no simulator, no matrix product over
the state):

* rz(phi) = diag(e^{-i phi/2}, e^{i phi/2})                    gates.rs:79-84
* u3(t, f, l) = [[cos t/2, -e^{il} sin t/2],
                 [e^{if} sin t/2, e^{i(f+l)} cos t/2]]         gates.rs:59-65
* u2(f, l) = u3(pi/2, f, l); u1 = p = diag(1, e^{il})          gates.rs:66-69
* rx(t) = [[c, -is], [-is, c]], ry(t) = [[c, -s], [s, c]]      gates.rs:71-78
* y = [[0, -i], [i, 0]], s, t, sx                              gates.rs:21-52
* two-qubit matrices are row-major with qubits[0] the most significant bit
  of the gate index: cp / crz / cu / cy = controlled(u) with the control
  first (gates.rs:121-143), rzz(t) = diag(e^-, e^+, e^+, e^-) (:155-160),
  rxx (:145-153)
* remote_link_psi_minus / psi_plus / phi_plus prepare the Bell states
  |Psi->, |Psi+>, |Phi+> from |00> (gates.rs:224-258), nonlocal_cz = cz
  (statevector/simulator.rs:582-584)
* rccx / rc3x / c3sqrtx phases (gates.rs:178-207)
* the QFT of a basis state |x> as this circuit writes it (h on qubit j, then
  cp(pi/2^(k-j)) controlled by every k > j, then swap(j, n-1-j)) ends in
  amp[w] = exp(2 pi i rev(x) rev(w) / 2^n) / 2^(n/2), rev = n-bit reversal
  (the phase of qubit j before the swaps is 2 pi rev(x) 2^j / 2^n).

State index bit q is qubit q (qubit 0 least significant), as in the
reference's ``Vec<Complex64>``.

Run: python tests/golden/make_amplitudes.py
"""
from __future__ import annotations

import cmath
import json
import math
from pathlib import Path

HERE = Path(__file__).resolve().parent
S = 1.0 / math.sqrt(2.0)


def ins(kind, **f):
    d = {"kind": kind}
    d.update(f)
    return d


def gen(name, qubits, params=()):
    return {"kind": "gate", "name": name, "params": list(params), "qubits": list(qubits)}


def fixture(name, n, instructions, amps, atol=1e-12):
    """amps: dict index -> complex (missing indices are exactly zero)."""
    vec = [[0.0, 0.0] for _ in range(1 << n)]
    for i, a in amps.items():
        vec[i] = [float(complex(a).real), float(complex(a).imag)]
    out = {
        "name": name,
        "num_qubits": n,
        "circuit": {"qregs": {"q": {"name": "q", "size": n, "base": 0}}, "cregs": {},
                    "instructions": instructions},
        "amplitudes": vec,
        "atol": atol,
    }
    (HERE / f"amp_{name}.json").write_text(json.dumps(out, indent=1) + "\n")


def e(phase):
    return cmath.exp(1j * phase)


def rev(v, n):
    r = 0
    for b in range(n):
        if (v >> b) & 1:
            r |= 1 << (n - 1 - b)
    return r


def main():
    h = lambda q: ins("h", qubit=q)
    x = lambda q: ins("x", qubit=q)

    # ---- one-qubit phase conventions ----
    phi = 0.7
    fixture("rz_plus", 1, [h(0), ins("rz", qubit=0, phi=phi)], {0: S * e(-phi / 2), 1: S * e(phi / 2)})
    t, f, l = 1.1, 0.4, 2.3
    fixture("u3_zero", 1, [ins("u3", qubit=0, theta=t, phi=f, lam=l)],
            {0: math.cos(t / 2), 1: e(f) * math.sin(t / 2)})
    fixture("u3_one", 1, [x(0), ins("u3", qubit=0, theta=t, phi=f, lam=l)],
            {0: -e(l) * math.sin(t / 2), 1: e(f + l) * math.cos(t / 2)})
    fixture("u_one", 1, [x(0), ins("u", qubit=0, theta=t, phi=f, lam=l)],
            {0: -e(l) * math.sin(t / 2), 1: e(f + l) * math.cos(t / 2)})
    fixture("u2_zero_one", 2, [x(1), ins("u2", qubit=0, phi=f, lam=l), ins("u2", qubit=1, phi=f, lam=l)],
            # q0: u2|0> = (1, e^{if})/sqrt2 ; q1: u2|1> = (-e^{il}, e^{i(f+l)})/sqrt2
            {0: S * -e(l) * S, 1: S * e(f) * S * -e(l), 2: S * e(f + l) * S,
             3: S * e(f) * S * e(f + l)})
    lam = 1.9
    fixture("u1_p_plus", 2, [h(0), h(1), ins("u1", qubit=0, lam=lam), ins("p", qubit=1, lam=-lam / 3)],
            {0: 0.5, 1: 0.5 * e(lam), 2: 0.5 * e(-lam / 3), 3: 0.5 * e(lam) * e(-lam / 3)})
    a, b = 0.9, 2.2
    ca, sa, cb, sb = math.cos(a / 2), math.sin(a / 2), math.cos(b / 2), math.sin(b / 2)
    fixture("rx_ry", 2, [ins("rx", qubit=0, theta=a), ins("ry", qubit=1, theta=b)],
            {0: ca * cb, 1: -1j * sa * cb, 2: ca * sb, 3: -1j * sa * sb})
    # sx|0> = ((1+i)/2, (1-i)/2); y|0> = i|1>; s h|0> = (1, i)/sqrt2; t h|0> = (1, e^{i pi/4})/sqrt2
    q0 = {0: (1 + 1j) / 2, 1: (1 - 1j) / 2}
    q1 = {0: 0.0, 1: 1j}
    q2 = {0: S, 1: 1j * S}
    q3 = {0: S, 1: S * e(math.pi / 4)}
    amps = {}
    for i in range(16):
        amps[i] = q0[i & 1] * q1[(i >> 1) & 1] * q2[(i >> 2) & 1] * q3[(i >> 3) & 1]
    fixture("sx_y_s_t", 4, [ins("sx", qubit=0), ins("y", qubit=1), h(2), ins("s", qubit=2), h(3),
                            ins("t", qubit=3)], amps)
    # sdg, tdg, sxdg: the conjugates
    q0 = {0: (1 - 1j) / 2, 1: (1 + 1j) / 2}
    q1 = {0: S, 1: -1j * S}
    q2 = {0: S, 1: S * e(-math.pi / 4)}
    amps = {i: q0[i & 1] * q1[(i >> 1) & 1] * q2[(i >> 2) & 1] for i in range(8)}
    fixture("sxdg_sdg_tdg", 3, [ins("sxdg", qubit=0), h(1), ins("sdg", qubit=1), h(2),
                                ins("tdg", qubit=2)], amps)

    # ---- two-qubit phase conventions (qubits[0] = MSB of the gate index) ----
    fixture("cp_plus", 2, [h(0), h(1), ins("cp", control=1, target=0, lam=lam)],
            {0: 0.5, 1: 0.5, 2: 0.5, 3: 0.5 * e(lam)})
    fixture("cu1_plus", 2, [h(0), h(1), ins("cu1", control=0, target=1, lam=-lam)],
            {0: 0.5, 1: 0.5, 2: 0.5, 3: 0.5 * e(-lam)})
    # crz(control 0, target 1): control set (index bit 0) -> rz(lam) on qubit 1
    fixture("crz_plus", 2, [h(0), h(1), ins("crz", control=0, target=1, lam=lam)],
            {0: 0.5, 2: 0.5, 1: 0.5 * e(-lam / 2), 3: 0.5 * e(lam / 2)})
    th = 1.3
    # rzz: e^{-i th/2} on even parity, e^{+i th/2} on odd parity
    fixture("rzz_plus", 2, [h(0), h(1), ins("rzz", a=0, b=1, theta=th)],
            {0: 0.5 * e(-th / 2), 3: 0.5 * e(-th / 2), 1: 0.5 * e(th / 2), 2: 0.5 * e(th / 2)})
    fixture("rxx_zero", 2, [ins("rxx", a=0, b=1, theta=th)],
            {0: math.cos(th / 2), 3: -1j * math.sin(th / 2)})
    # rxx(a=1, b=0) on |q0=1, q1=0>: qubits[0] = a = q1 is the MSB, so the gate
    # index is 2*0 + 1 = 1 and column 1 is (0, c, -is, 0): gate index 1
    # (q1=0, q0=1) -> state index 1, gate index 2 (q1=1, q0=0) -> state index 2
    fixture("rxx_swapped_order", 2, [x(0), ins("rxx", a=1, b=0, theta=th)],
            {1: math.cos(th / 2), 2: -1j * math.sin(th / 2)})
    g_ = 0.6
    # cu on |control=1, target=0>: e^{i gamma} u3(t,f,l)|0>
    fixture("cu_gamma", 2, [x(0), ins("cu", control=0, target=1, theta=t, phi=f, lam=l, gamma=g_)],
            {1: e(g_) * math.cos(t / 2), 3: e(g_ + f) * math.sin(t / 2)})
    fixture("cu3_one", 2, [x(0), x(1), ins("cu3", control=0, target=1, theta=t, phi=f, lam=l)],
            {1: -e(l) * math.sin(t / 2), 3: e(f + l) * math.cos(t / 2)})
    fixture("cy_one", 2, [x(0), ins("cy", control=0, target=1)], {3: 1j})
    fixture("cy_one_one", 2, [x(0), x(1), ins("cy", control=0, target=1)], {1: -1j})
    fixture("crx_cry", 3, [x(0), ins("crx", control=0, target=1, theta=a),
                           ins("cry", control=0, target=2, theta=b)],
            {1: ca * cb, 3: -1j * sa * cb, 5: ca * sb, 7: -1j * sa * sb})
    fixture("ch_csx", 3, [x(2), ins("ch", control=2, target=0), ins("csx", control=2, target=1)],
            # q0: h|0> = (1, 1)/sqrt2 ; q1: sx|0> = ((1+i)/2, (1-i)/2) ; q2 = 1
            {4: S * (1 + 1j) / 2, 5: S * (1 + 1j) / 2, 6: S * (1 - 1j) / 2, 7: S * (1 - 1j) / 2})

    # ---- remote-link gates: Bell-state preparation from |00> ----
    fixture("psi_minus_bell", 2, [gen("remote_link_psi_minus", [0, 1])], {2: S, 1: -S})
    fixture("psi_plus_bell", 2, [gen("remote_link_psi_plus", [0, 1])], {2: S, 1: S})
    fixture("phi_plus_bell", 2, [gen("remote_link_phi_plus", [0, 1])], {0: S, 3: S})
    # on |q0=1, q1=1> (gate index 3): columns 3 of the matrices
    fixture("psi_minus_11", 2, [x(0), x(1), gen("remote_link_psi_minus", [0, 1])], {0: S, 3: S})
    fixture("psi_plus_11", 2, [x(0), x(1), gen("remote_link_psi_plus", [0, 1])], {0: S, 3: -S})
    fixture("phi_plus_11", 2, [x(0), x(1), gen("remote_link_phi_plus", [0, 1])], {2: S, 1: -S})
    # reversed qubit order: qubits [1, 0] -> qubits[0] = q1 is the MSB; on |q0=1, q1=0>
    # the gate index is 2*0 + 1 = 1: psi_minus column 1 = (s, 0, 0, -s)
    fixture("psi_minus_rev", 2, [x(0), gen("remote_link_psi_minus", [1, 0])], {0: S, 3: -S})
    fixture("nonlocal_cz_plus", 2, [h(0), h(1), gen("nonlocal_cz", [0, 1])],
            {0: 0.5, 1: 0.5, 2: 0.5, 3: -0.5})

    # ---- multi-controlled phases ----
    # rccx(c1=0, c2=1, t=2) on |c1=1, c2=1, t=0>: gate index 6 -> m[7][6] = -i
    fixture("rccx_phase", 3, [x(0), x(1), ins("rccx", control1=0, control2=1, target=2)], {7: -1j})
    # rc3x(c=0,1,2; t=3) on controls set, target 0: gate index 14 -> m[14][14] = i
    fixture("rc3x_phase", 4, [x(0), x(1), x(2),
                              ins("rc3x", control1=0, control2=1, control3=2, target=3)], {7: 1j})
    # c3sqrtx on controls set, target 0: sx|0> on the target
    fixture("c3sqrtx_one", 4, [x(0), x(1), x(2),
                               ins("c3sqrtx", control1=0, control2=1, control3=2, target=3)],
            {7: (1 + 1j) / 2, 15: (1 - 1j) / 2})

    # ---- QFT of basis states: every phase of the cp ladder ----
    for n, xbits in ((5, 0b10110), (6, 0b000001), (8, 0b11100101)):
        insts = [x(q) for q in range(n) if xbits >> q & 1]
        for j in range(n):
            insts.append(h(j))
            for k in range(j + 1, n):
                insts.append(ins("cp", control=k, target=j, lam=math.pi / 2 ** (k - j)))
        for j in range(n // 2):
            insts.append(ins("swap", a=j, b=n - 1 - j))
        N = 1 << n
        rx_ = rev(xbits, n)
        amps = {w: e(2 * math.pi * ((rx_ * rev(w, n)) % N) / N) / math.sqrt(N) for w in range(N)}
        fixture(f"qft{n}_basis_{xbits}", n, insts, amps)


if __name__ == "__main__":
    main()
