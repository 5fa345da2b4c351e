"""Writes the golden fixtures of this directory.

Each fixture is a circuit in the bosonic-model JSON layout that the
reference decodes (src/types.rs:8-135) plus its exact, closed-form output
distribution.  The circuits are the ones the reference's own tests pin the
statevector path with (tests/test_distribution_e2e.py:167-216, tolerance
1e-6; tests/test_qasmbench_simulation.py:91-93, norm 1e-6); the expected
values are computed analytically below, not by any simulator.  The QFT of a
basis state has the uniform distribution 2^-n for every input.

Run: python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
from pathlib import Path

HERE = Path(__file__).resolve().parent


def ins(kind, **f):
    d = {"kind": kind}
    d.update(f)
    return d


def circuit(n, instructions):
    return {"qregs": {"q": {"name": "q", "size": n, "base": 0}}, "cregs": {},
            "instructions": instructions}


def fixture(name, n, instructions, probs, atol=1e-12):
    out = {
        "name": name,
        "num_qubits": n,
        "circuit": circuit(n, instructions),
        "probabilities": {str(k): v for k, v in sorted(probs.items())},
        "atol": atol,
        "seed": 42,
    }
    (HERE / f"{name}.json").write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")


def main():
    h = lambda q: ins("h", qubit=q)
    x = lambda q: ins("x", qubit=q)
    cx = lambda c, t: ins("cx", control=c, target=t)
    fixture("bell_pair", 2, [h(0), cx(0, 1)], {0: 0.5, 3: 0.5})
    fixture("x_cx_deterministic", 2, [x(0), cx(0, 1)], {3: 1.0})
    fixture("cz_pair", 2, [h(0), h(1), ins("cz", control=0, target=1)], {i: 0.25 for i in range(4)})
    c6, s6 = math.cos(math.pi / 6) ** 2, math.sin(math.pi / 6) ** 2
    fixture("ry_cx", 2, [ins("ry", qubit=0, theta=math.pi / 3), cx(0, 1)], {0: c6, 3: s6})
    c8, s8 = math.cos(math.pi / 8) ** 2, math.sin(math.pi / 8) ** 2
    fixture("rx_ry_cx", 2, [ins("rx", qubit=0, theta=math.pi / 3),
                            ins("ry", qubit=1, theta=math.pi / 4), cx(0, 1)],
            {0: c6 * c8, 1: s6 * s8, 2: c6 * s8, 3: s6 * c8})
    fixture("xyz_single", 2, [x(0), ins("y", qubit=1), ins("z", qubit=0)], {3: 1.0})
    fixture("local_hh", 2, [h(0), h(1)], {i: 0.25 for i in range(4)})
    fixture("ghz4", 4, [h(0), cx(0, 1), cx(1, 2), cx(2, 3)], {0: 0.5, 15: 0.5})
    # h q0; cx 0->2; cx 1->3: q0 and q2 perfectly correlated, q1 = q3 = 0
    fixture("chain_cx4", 4, [h(0), cx(0, 2), cx(1, 3)], {0: 0.5, 5: 0.5})
    fixture("local_4h", 4, [h(q) for q in range(4)], {i: 1 / 16 for i in range(16)})
    # QFT of basis states: |amplitude|^2 = 2^-n for every output
    for n, xbits in ((5, 0b10110), (6, 0b000001), (8, 0b11100101)):
        insts = [x(q) for q in range(n) if xbits >> q & 1]
        for j in range(n):
            insts.append(h(j))
            for k in range(j + 1, n):
                insts.append(ins("cp", control=k, target=j, lam=math.pi / 2 ** (k - j)))
        for j in range(n // 2):
            insts.append(ins("swap", a=j, b=n - 1 - j))
        fixture(f"qft{n}_basis_{xbits}", n, insts, {i: 2.0 ** -n for i in range(2 ** n)})


if __name__ == "__main__":
    main()
