"""ctypes binding of ``libdqsim_cuda.so`` (the C ABI in ``include/dqsim_cuda.h``).

The library is the only compute path of this package.  If it is missing or
cannot be loaded, every simulation call raises instead of falling back to
anything else.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("DQSIM_CUDA_LIB", _PKG / "libdqsim_cuda.so"))

# ---- status codes (include/dqsim_cuda.h) -------------------------------------
DQ_OK = 0
DQ_ERR_INVALID_ARG = -1
DQ_ERR_CUDA = -2
DQ_ERR_OOM = -3
DQ_ERR_UNSUPPORTED = -4
DQ_ERR_NO_DEVICE = -5
DQ_ERR_INTERNAL = -6
DQ_ERR_DECODE = -7

# ---- instruction kinds (enum dq_kind) --------------------------------------------
KIND_NAMES = [
    "id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg",
    "u3", "u2", "u1", "u", "p", "rx", "ry", "rz", "u0",
    "cx", "cz", "cy", "ch", "swap", "csx",
    "crx", "cry", "crz", "cu1", "cp", "cu3", "cu", "rxx", "rzz",
    "ccx", "cswap", "rccx", "rc3x", "c3x", "c3sqrtx", "c4x",
    "g_phi_plus", "g_psi_minus", "g_psi_plus", "g_cz", "g_cx", "g_noop", "g_opaque",
    "g_unsupported",
    "measure", "reset", "barrier", "classical",
]
KIND = {name: i for i, name in enumerate(KIND_NAMES)}
MAX_INST_QUBITS = 8

SEM_SIMULATE = 0
SEM_SHOTS = 1
EXEC_PER_GATE = 0
EXEC_FUSED = 1

# dq_inst / dq_cond as numpy record layouts (C struct alignment)
INST_DTYPE = np.dtype(
    [
        ("kind", "<i4"),
        ("nq", "<i4"),
        ("q", "<i4", (MAX_INST_QUBITS,)),
        ("cbit", "<i8"),
        ("p", "<f8", (4,)),
        ("cond_first", "<u4"),
        ("cond_count", "<u4"),
    ],
    align=True,
)
COND_DTYPE = np.dtype([("creg_base", "<u8"), ("creg_size", "<u8"), ("creg_value", "<u8")], align=True)
PAULI_DTYPE = np.dtype([("coeff", "<f8"), ("xmask", "<u8"), ("zmask", "<u8")], align=True)
assert INST_DTYPE.itemsize == 88 and COND_DTYPE.itemsize == 24 and PAULI_DTYPE.itemsize == 24


class RunOpts(ctypes.Structure):
    _fields_ = [
        ("semantics", ctypes.c_int32),
        ("exec", ctypes.c_int32),
        ("fusion_width", ctypes.c_int32),
        ("profile", ctypes.c_int32),
        ("time_sweeps", ctypes.c_int32),
        ("max_cost", ctypes.c_int32),
    ]


class Profile(ctypes.Structure):
    _fields_ = [
        ("apply_one_qubit_calls", ctypes.c_uint64),
        ("apply_one_qubit_time", ctypes.c_double),
        ("apply_n_qubit_calls", ctypes.c_uint64),
        ("apply_n_qubit_time", ctypes.c_double),
        ("measure_qubit_calls", ctypes.c_uint64),
        ("measure_qubit_time", ctypes.c_double),
        ("total_time", ctypes.c_double),
        ("kernel_launches", ctypes.c_uint64),
        ("sweeps", ctypes.c_uint64),
        ("sweep_time", ctypes.c_double),
        ("boundary_draws", ctypes.c_uint64),
        ("failed_inst", ctypes.c_int64),
    ]


class TrajOpts(ctypes.Structure):
    _fields_ = [
        ("threads", ctypes.c_int32),
        ("max_cluster", ctypes.c_int32),
        ("local_bits", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class MpsStats(ctypes.Structure):
    _fields_ = [
        ("svd_calls", ctypes.c_uint64),
        ("kernel_ms", ctypes.c_double),
        ("failed_inst", ctypes.c_int64),
        ("capacity", ctypes.c_uint32),
        ("replicas", ctypes.c_uint32),
    ]


class TrajStats(ctypes.Structure):
    _fields_ = [
        ("boundary_draws", ctypes.c_uint64),
        ("failed_inst", ctypes.c_int64),
        ("kernel_ms", ctypes.c_double),
        ("prepare_ms", ctypes.c_double),
        ("engine_ms", ctypes.c_double),
        ("cluster_span", ctypes.c_uint32),
        ("clusters", ctypes.c_uint32),
        ("threads", ctypes.c_uint32),
        ("local_bits", ctypes.c_uint32),
        ("launches", ctypes.c_uint32),
        ("engine_items", ctypes.c_uint32),
        ("hbm_items", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class AdjointBatchStats(ctypes.Structure):
    _fields_ = [
        ("launches", ctypes.c_uint64),
        ("forward_sweeps", ctypes.c_uint64),
        ("backward_sweeps", ctypes.c_uint64),
        ("plan_ms", ctypes.c_double),
        ("forward_ms", ctypes.c_double),
        ("observable_ms", ctypes.c_double),
        ("backward_ms", ctypes.c_double),
        ("batched", ctypes.c_uint32),
        ("groups", ctypes.c_uint32),
    ]


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("prog", ctypes.c_void_p),
        ("ninst", ctypes.c_uint64),
        ("conds", ctypes.c_void_p),
        ("nconds", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("cbits_out", ctypes.c_void_p),
        ("ncbits", ctypes.c_uint64),
        ("state_out", ctypes.c_void_p),
    ]


class CircuitInfo(ctypes.Structure):
    _fields_ = [
        ("ninst", ctypes.c_uint64),
        ("ncond", ctypes.c_uint64),
        ("num_qubits", ctypes.c_uint64),
        ("num_cbits", ctypes.c_uint64),
        ("cbit_space", ctypes.c_uint64),
        ("names_bytes", ctypes.c_uint64),
    ]


class EngineError(RuntimeError):
    """A non-OK status returned by the engine."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class UnsupportedGate(EngineError):
    pass


_P = ctypes.c_void_p
_U32 = ctypes.c_uint32
_U64 = ctypes.c_uint64
_I32 = ctypes.c_int32
_DP = ctypes.POINTER(ctypes.c_double)

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("dq_abi_version", ctypes.c_int, []),
    ("dq_last_error", ctypes.c_char_p, []),
    ("dq_device_count", ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    ("dq_circuit_decode", ctypes.c_int, [ctypes.c_char_p, _U64, ctypes.POINTER(_P),
                                         ctypes.POINTER(CircuitInfo)]),
    ("dq_circuit_export", ctypes.c_int, [_P, _P, _P, _P]),
    ("dq_circuit_free", None, [_P]),
    ("dq_state_create", ctypes.c_int, [_U32, ctypes.c_int, ctypes.POINTER(_P)]),
    ("dq_state_destroy", ctypes.c_int, [_P]),
    ("dq_state_num_qubits", ctypes.c_int, [_P, ctypes.POINTER(_U32)]),
    ("dq_state_reset", ctypes.c_int, [_P]),
    ("dq_state_set_basis", ctypes.c_int, [_P, _U64]),
    ("dq_state_upload", ctypes.c_int, [_P, _P, _U64]),
    ("dq_state_download", ctypes.c_int, [_P, _P, _U64]),
    ("dq_state_copy", ctypes.c_int, [_P, _P]),
    ("dq_state_device_ptr", ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    ("dq_state_synchronize", ctypes.c_int, [_P]),
    ("dq_apply_1q", ctypes.c_int, [_P, _P, _U32, _U64, _U64]),
    ("dq_apply_dense", ctypes.c_int, [_P, _P, _P, _U32]),
    ("dq_apply_inst", ctypes.c_int, [_P, _P]),
    ("dq_measure_p1", ctypes.c_int, [_P, _U32, _DP]),
    ("dq_collapse", ctypes.c_int, [_P, _U32, ctypes.c_int, ctypes.c_double]),
    ("dq_measure", ctypes.c_int, [_P, _U32, ctypes.c_double, ctypes.POINTER(ctypes.c_int), _DP]),
    ("dq_measure_p1_noalloc", ctypes.c_int, [_P, _U32, _U32, _P, _P]),
    ("dq_run", ctypes.c_int, [_P, _P, _U64, _P, _U64, _U64, _P, _U64, ctypes.POINTER(RunOpts),
                              ctypes.POINTER(Profile)]),
    ("dq_marginal_probs", ctypes.c_int, [_P, _P, _U32, _P]),
    ("dq_sample", ctypes.c_int, [_P, _P, _U32, _U64, _U64, _P, ctypes.POINTER(_U64)]),
    ("dq_sample_key", ctypes.c_int, [_P, _P, _U32, _P, _U64, _P, ctypes.POINTER(_U64)]),
    ("dq_inner", ctypes.c_int, [_P, _P, _U64, _DP, _DP]),
    ("dq_norm_sqr", ctypes.c_int, [_P, _DP]),
    ("dq_run_trajectories", ctypes.c_int, [ctypes.c_int, _U32, _P, _U64, _P, _U64, _U64, _U64,
                                           _U64, _P, _U64, ctypes.POINTER(TrajOpts),
                                           ctypes.POINTER(TrajStats)]),
    ("dq_traj_plan_create", ctypes.c_int, [ctypes.c_int, _U32, _P, _U64, _P, _U64, _U64, _U64,
                                           ctypes.POINTER(TrajOpts), ctypes.POINTER(_P)]),
    ("dq_traj_plan_run", ctypes.c_int, [_P, _U64, _P, ctypes.POINTER(TrajStats)]),
    ("dq_traj_plan_destroy", ctypes.c_int, [_P]),
    ("dq_run_batch", ctypes.c_int, [ctypes.c_int, _P, _U64, ctypes.POINTER(TrajOpts),
                                    ctypes.POINTER(TrajStats)]),
    ("dq_expval_pauli", ctypes.c_int, [_P, _P, _U64, _DP]),
    ("dq_adjoint", ctypes.c_int, [_P, _P, _U64, _P, _U64, _P, _U64, ctypes.POINTER(RunOpts), _DP,
                                  _P, _P]),
    ("dq_adjoint_batch", ctypes.c_int, [ctypes.c_int, _U32, _P, _U64, _P, _U64, _P, _U64, _P, _U64,
                                        _P, _P, ctypes.POINTER(AdjointBatchStats)]),
    ("dq_debug_plan", ctypes.c_int, [_U32, _P, _U64, ctypes.POINTER(RunOpts), _P, _U64,
                                     ctypes.POINTER(_U64)]),
    ("dq_block_merge", ctypes.c_int, [_P, _P, _U32, _P, _P, _U32, _P]),
    ("dq_mps_create", ctypes.c_int, [_U32, ctypes.c_int, _U32, ctypes.c_double, ctypes.POINTER(_P)]),
    ("dq_mps_destroy", ctypes.c_int, [_P]),
    ("dq_mps_run", ctypes.c_int, [_P, _P, _U64, _P, _U64, _U64, _P, _U64,
                                  ctypes.POINTER(MpsStats)]),
    ("dq_mps_apply_2q", ctypes.c_int, [_P, _U32, _U32, _P]),
    ("dq_mps_reserve", ctypes.c_int, [_P, _U32]),
    ("dq_mps_bond_dims", ctypes.c_int, [_P, _P]),
    ("dq_mps_to_state", ctypes.c_int, [_P, _P]),
    ("dq_mps_run_shots", ctypes.c_int, [ctypes.c_int, _U32, _U32, ctypes.c_double, _P, _U64, _P,
                                        _U64, _U64, _U64, _U64, _P, _U64, _U32,
                                        ctypes.POINTER(MpsStats)]),
    ("dq_rng_f64", ctypes.c_int, [_U64, _U64, _U64, _P]),
    ("dq_rng_seed_key", ctypes.c_int, [_U64, _P]),
    ("dq_chacha_block", ctypes.c_int, [_P, _U32, _P]),
]

_lib = None


def lib():
    """Load (once) and return the engine library; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"dqsim engine library not found at {LIB_PATH}; build it with "
            "`python -m dqsim_bosonic_b200.build` (nvcc, sm_100a)"
        )
    L = ctypes.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if L.dq_abi_version() != 1:
        raise ImportError("libdqsim_cuda.so ABI version mismatch")
    _lib = L
    return L


def last_error() -> str:
    msg = lib().dq_last_error()
    return msg.decode("utf-8", "replace") if msg else ""


def check(rc: int, what: str = "") -> None:
    if rc == DQ_OK:
        return
    msg = last_error()
    text = f"{what}: {msg}" if what else msg
    if rc == DQ_ERR_UNSUPPORTED:
        raise UnsupportedGate(rc, text)
    if rc == DQ_ERR_INVALID_ARG:
        raise ValueError(text)
    if rc == DQ_ERR_OOM:
        raise MemoryError(text)
    raise EngineError(rc, text)


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def device_count() -> int:
    c = ctypes.c_int(0)
    rc = lib().dq_device_count(ctypes.byref(c))
    if rc != DQ_OK:
        return 0
    return c.value


class State:
    """Owning wrapper of a ``dq_state_t`` (a 2^n complex128 vector in HBM)."""

    def __init__(self, n: int, device: int = 0):
        L = lib()
        h = _P()
        check(L.dq_state_create(int(n), int(device), ctypes.byref(h)), "dq_state_create")
        self._h = h
        self.n = int(n)
        self.device = int(device)

    @property
    def handle(self):
        if self._h is None:
            raise ValueError("state was released")
        return self._h

    def release(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib().dq_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def reset(self) -> None:
        check(lib().dq_state_reset(self.handle), "dq_state_reset")

    def set_basis(self, index: int) -> None:
        check(lib().dq_state_set_basis(self.handle, int(index)), "dq_state_set_basis")

    def download(self) -> np.ndarray:
        out = np.empty(1 << self.n, dtype=np.complex128)
        check(lib().dq_state_download(self.handle, ptr(out), out.size), "dq_state_download")
        return out

    def upload(self, amps: np.ndarray) -> None:
        a = np.ascontiguousarray(amps, dtype=np.complex128)
        check(lib().dq_state_upload(self.handle, ptr(a), a.size), "dq_state_upload")

    def device_ptr(self) -> tuple[int, int]:
        p, s = _P(), _P()
        check(lib().dq_state_device_ptr(self.handle, ctypes.byref(p), ctypes.byref(s)))
        return p.value or 0, s.value or 0
