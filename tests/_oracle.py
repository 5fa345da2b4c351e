"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is test infrastructure: a C restatement of the reference's
statevector engine (see oracle/oracle.c).  Tests use it as the checker only.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

_lib = None


def build_oracle() -> Path:
    src = ORACLE_DIR / "oracle.c"
    if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-C", str(ORACLE_DIR)], check=True, capture_output=True)
    return ORACLE_LIB


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(str(ORACLE_LIB))
        P, U32, U64, I64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int64
        sig = {
            "or_set_threads": (None, [ctypes.c_int]),
            "or_get_max_threads": (ctypes.c_int, []),
            "or_chacha_block": (None, [P, U32, P]),
            "or_seed_key": (None, [U64, P]),
            "or_rng_f64_stream": (None, [U64, U64, U64, P]),
            "or_apply_one_qubit": (None, [P, U32, P, U32, U64, U64]),
            "or_apply_n_qubit": (None, [P, U32, P, P, U32]),
            "or_p1": (ctypes.c_double, [P, U32, U32]),
            "or_measure": (ctypes.c_int, [P, U32, U32, ctypes.c_double, P]),
            "or_marginal_probs": (None, [P, U32, P, U32, P]),
            "or_sample": (None, [P, U32, P, U32, U64, U64, P]),
            "or_matrix_1q": (ctypes.c_int, [ctypes.c_int, P, P]),
            "or_matrix_nq": (ctypes.c_int, [P, P, P]),
            "or_run": (ctypes.c_int, [P, U32, P, U64, P, U64, P, U64, P]),
            "or_run_shots": (ctypes.c_int, [U32, P, U64, P, U64, U64, U64, P, U64, P]),
            "or_fuse_export": (U64, [P, U64, U32, P, P, P]),
            "or_expval_pauli": (ctypes.c_double, [P, U32, P, U64]),
            "or_block_merge": (U32, [P, P, U32, P, P, U32, P]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def set_threads(t: int) -> None:
    lib().or_set_threads(int(t))


def chacha_block(in16: np.ndarray, rounds: int) -> np.ndarray:
    a = np.ascontiguousarray(in16, dtype=np.uint32)
    out = np.empty(16, dtype=np.uint32)
    lib().or_chacha_block(_p(a), rounds, _p(out))
    return out


def seed_key(seed: int) -> np.ndarray:
    out = np.empty(8, dtype=np.uint32)
    lib().or_seed_key(seed, _p(out))
    return out


def rng_f64(seed: int, skip: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    lib().or_rng_f64_stream(seed, skip, count, _p(out))
    return out


def run(prog, seed: int, init: np.ndarray | None = None):
    """simulate(): returns (statevector, cbits array, rc, failed index)."""
    n = prog.num_qubits
    st = np.zeros(1 << n, dtype=np.complex128)
    if init is None:
        st[0] = 1.0
    else:
        st[:] = init
    cbits = np.full(prog.cbit_space, -1, dtype=np.int32)
    failed = ctypes.c_int64(-1)
    rc = lib().or_run(_p(st), n, _p(prog.insts), prog.ninst,
                      _p(prog.conds) if prog.conds.size else None, seed & ((1 << 64) - 1),
                      _p(cbits), cbits.size, ctypes.byref(failed))
    return st, cbits, rc, failed.value


def run_inplace(prog, seed: int, state: np.ndarray) -> int:
    """Run prog on state (complex128, modified in place); returns the status."""
    cbits = np.full(max(prog.cbit_space, 1), -1, dtype=np.int32)
    failed = ctypes.c_int64(-1)
    return lib().or_run(_p(state), prog.num_qubits, _p(prog.insts), prog.ninst,
                        _p(prog.conds) if prog.conds.size else None, seed & ((1 << 64) - 1),
                        _p(cbits), cbits.size, ctypes.byref(failed))


def run_shots(prog, base_seed: int, shots: int, shot0: int = 0):
    cb = np.full((shots, prog.cbit_space), -1, dtype=np.int32)
    failed = ctypes.c_int64(-1)
    rc = lib().or_run_shots(prog.num_qubits, _p(prog.insts), prog.ninst,
                            _p(prog.conds) if prog.conds.size else None, base_seed & ((1 << 64) - 1),
                            shot0, shots, _p(cb), prog.cbit_space, ctypes.byref(failed))
    return cb, rc, failed.value


def marginal(state: np.ndarray, qubits) -> np.ndarray:
    n = int(state.size).bit_length() - 1
    q = np.asarray(qubits, dtype=np.uint32)
    out = np.empty(1 << len(q), dtype=np.float64)
    s = np.ascontiguousarray(state)
    lib().or_marginal_probs(_p(s), n, _p(q) if q.size else None, len(q), _p(out))
    return out


def sample(state: np.ndarray, qubits, seed: int, shots: int) -> np.ndarray:
    n = int(state.size).bit_length() - 1
    q = np.asarray(qubits, dtype=np.uint32)
    out = np.empty(max(shots, 1), dtype=np.uint32)
    s = np.ascontiguousarray(state)
    lib().or_sample(_p(s), n, _p(q) if q.size else None, len(q), seed, shots, _p(out))
    return out[:shots]


def apply_one_qubit(state: np.ndarray, u: np.ndarray, target: int, incl: int = 0, desired: int = 0):
    n = int(state.size).bit_length() - 1
    um = np.ascontiguousarray(u, dtype=np.complex128).reshape(4)
    lib().or_apply_one_qubit(_p(state), n, _p(um), target, incl, desired)


def apply_n_qubit(state: np.ndarray, u: np.ndarray, qubits) -> None:
    n = int(state.size).bit_length() - 1
    q = np.asarray(qubits, dtype=np.uint32)
    um = np.ascontiguousarray(u, dtype=np.complex128)
    lib().or_apply_n_qubit(_p(state), n, _p(um), _p(q), len(q))


def p1(state: np.ndarray, q: int) -> float:
    n = int(state.size).bit_length() - 1
    return lib().or_p1(_p(state), n, q)


def measure(state: np.ndarray, q: int, r: float) -> tuple[int, float]:
    n = int(state.size).bit_length() - 1
    pp = ctypes.c_double(0.0)
    o = lib().or_measure(_p(state), n, q, r, ctypes.byref(pp))
    return o, pp.value


def fuse(prog):
    n = prog.num_qubits
    cap = prog.ninst + n + 1
    inst = np.empty(cap, dtype=np.int64)
    qub = np.empty(cap, dtype=np.uint32)
    mat = np.empty((cap, 4), dtype=np.complex128)
    nf = lib().or_fuse_export(_p(prog.insts), prog.ninst, n, _p(inst), _p(qub), _p(mat))
    return inst[:nf], qub[:nf], mat[:nf]


def expval_pauli(state: np.ndarray, terms: np.ndarray) -> float:
    """<psi|H|psi> on the CPU for a PAULI_DTYPE term array."""
    st = np.ascontiguousarray(state, dtype=np.complex128)
    t = np.ascontiguousarray(terms)
    n = int(st.size).bit_length() - 1
    return float(lib().or_expval_pauli(_p(st), n, _p(t), len(t)))


def run_unitary(insts: np.ndarray, n: int, init: np.ndarray | None = None) -> np.ndarray:
    """Final state of a unitary dq_inst program on the CPU (from |0> or init)."""
    st = np.zeros(1 << n, dtype=np.complex128)
    if init is None:
        st[0] = 1.0
    else:
        st[:] = init
    cb = np.full(1, -1, dtype=np.int32)
    failed = ctypes.c_int64(-1)
    a = np.ascontiguousarray(insts)
    rc = lib().or_run(_p(st), n, _p(a), len(a), None, 0, _p(cb), 1, ctypes.byref(failed))
    if rc != 0:
        raise RuntimeError(f"oracle run failed: {rc}")
    return st


def expval_program(insts: np.ndarray, n: int, terms: np.ndarray) -> float:
    return expval_pauli(run_unitary(insts, n), terms)


# Shift rules restated for the checker: two-term rule for generators with a
# single eigenvalue gap of 1 (rx/ry/rz/rxx/rzz, phases, u3 angles), four-term
# rule (gaps 1/2 and 1) for controlled rotations.
_R2 = ((0.5, np.pi / 2), (-0.5, -np.pi / 2))
_d1 = (np.sqrt(2) + 1) / (4 * np.sqrt(2))
_d2 = (np.sqrt(2) - 1) / (4 * np.sqrt(2))
_R4 = ((_d1, np.pi / 2), (-_d1, -np.pi / 2), (-_d2, 3 * np.pi / 2), (_d2, -3 * np.pi / 2))


def param_shift(circuit, theta, terms: np.ndarray, occurrences=None) -> np.ndarray:
    """Parameter-shift gradient with every forward run on the oracle."""
    base = circuit.bind(theta)
    n = circuit.num_qubits
    occ = circuit.occurrences()
    grad = np.zeros(circuit.num_params)
    for o in (range(len(occ)) if occurrences is None else occurrences):
        i, j, p = occ[o]
        kind = circuit.ops[i][0]
        rule = _R4 if (kind in ("crx", "cry", "crz") or (kind in ("cu3", "cu") and j == 0)) else _R2
        g = 0.0
        for c, s in rule:
            a = base.copy()
            a[i]["p"][j] += s
            g += c * expval_program(a, n, terms)
        grad[p.index] += p.scale * g
    return grad


def finite_difference(circuit, theta, terms: np.ndarray, h: float = 1e-6, entries=None) -> np.ndarray:
    """Central differences of <H> in theta on the oracle."""
    th = np.asarray(theta, dtype=np.float64).copy()
    n = circuit.num_qubits
    out = np.zeros(th.size)
    for k in (range(th.size) if entries is None else entries):
        tp = th.copy(); tp[k] += h
        tm = th.copy(); tm[k] -= h
        out[k] = (expval_program(circuit.bind(tp), n, terms) -
                  expval_program(circuit.bind(tm), n, terms)) / (2 * h)
    return out


def block_merge(a: np.ndarray, qa, b: np.ndarray, qb) -> tuple[np.ndarray, list[int]]:
    """merge_blocks on the CPU: (merged state, merged qubits)."""
    qa = np.ascontiguousarray(qa, dtype=np.uint32)
    qb = np.ascontiguousarray(qb, dtype=np.uint32)
    u = sorted(set(qa.tolist()) | set(qb.tolist()))
    out = np.empty(1 << len(u), dtype=np.complex128)
    a = np.ascontiguousarray(a, dtype=np.complex128)
    b = np.ascontiguousarray(b, dtype=np.complex128)
    n = lib().or_block_merge(_p(a), _p(qa) if qa.size else None, qa.size, _p(b),
                             _p(qb) if qb.size else None, qb.size, _p(out))
    assert n == len(u)
    return out, u


def _load_mps_oracle():
    import importlib.util
    spec = importlib.util.spec_from_file_location("oracle_mps", ORACLE_DIR / "mps.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


_mps_mod = None


def mps_module():
    global _mps_mod
    if _mps_mod is None:
        _mps_mod = _load_mps_oracle()
    return _mps_mod


class _Draws:
    """Sequential gen::<f64>() draws of ChaCha8Rng::seed_from_u64(seed)."""

    def __init__(self, seed: int):
        self.seed = seed
        self.pos = 0
        self.buf = np.zeros(0)
        self.base = 0

    def __call__(self) -> float:
        if self.pos - self.base >= self.buf.size:
            self.base = self.pos
            self.buf = rng_f64(self.seed, self.pos, 256)
        v = float(self.buf[self.pos - self.base])
        self.pos += 1
        return v


def _mps_classify(rec):
    from dqsim_bosonic_b200._native import KIND
    kind = int(rec["kind"])
    if kind in (KIND["id"], KIND["u0"], KIND["barrier"], KIND["classical"], KIND["g_noop"],
                KIND["g_opaque"]):
        return "noop", None
    if kind == KIND["measure"]:
        return "measure", None
    if kind == KIND["reset"]:
        return "reset", None
    m = np.zeros(4, dtype=np.complex128)
    p = np.ascontiguousarray(rec["p"], dtype=np.float64)
    if lib().or_matrix_1q(kind, _p(p), _p(m)):
        return "1q", m.reshape(2, 2)
    big = np.zeros(32 * 32, dtype=np.complex128)
    qs = np.zeros(8, dtype=np.uint32)
    r = np.array([rec])
    k = lib().or_matrix_nq(_p(r), _p(big), _p(qs))
    if k == 2:
        return "2q", big[:16].reshape(4, 4).copy()
    return "fail", None


def mps_run(prog, seed: int, max_bond=None, threshold: float = 1e-12):
    """The MPS oracle over an encoded program: (statevector, cbits, bond dims, svd calls)."""
    mod = mps_module()
    mps, cbits = mod.run(prog.insts, prog.conds, prog.num_qubits, prog.cbit_space, _Draws(seed),
                         _mps_classify, max_bond, threshold)
    return mps.to_statevector(), cbits, mps.bond_dims(), mps.svd_calls
