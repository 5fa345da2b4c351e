"""Host-side logic with no GPU: JSON decoding, IR encoding, mode parsing, ABI.

The codecs tests mirror the reference's tests/test_codecs.py: mode and
options are parsed before the circuit is touched, which an ``object()``
without ``model_dump_json`` proves.
"""
import ctypes
import json
import math
import re
from pathlib import Path

import numpy as np
import pytest

from _circuits import JsonCircuit, cond, g, gate
from dqsim_bosonic_b200 import simulate_distributed, simulate_monolithic, simulate_monolithic_shots
from dqsim_bosonic_b200 import _native as nat
from dqsim_bosonic_b200.circuit import (CircuitDecodeError, decode_circuit_json, encode,
                                        format_cbits)

ROOT = Path(__file__).resolve().parents[1]


# ---- codecs (reference tests/test_codecs.py) -------------------------------------------


@pytest.mark.parametrize("mode", ["state_vector", "state-vector", "statevector", "sv", " SV "])
def test_statevector_mode_aliases_are_accepted_before_circuit_decoding(mode):
    with pytest.raises(AttributeError, match="model_dump_json"):
        simulate_monolithic(object(), mode=mode)


@pytest.mark.parametrize("mode", ["mps", "matrix_product_state", "matrix-product-state", " MPS "])
def test_mps_mode_aliases_are_accepted_before_circuit_decoding(mode):
    with pytest.raises(AttributeError, match="model_dump_json"):
        simulate_monolithic(object(), mode=mode)


def test_invalid_monolithic_mode_raises():
    with pytest.raises(ValueError, match="Unsupported monolithic simulation mode"):
        simulate_monolithic(object(), mode="tensor_network")


def test_statevector_mode_rejects_mps_options():
    with pytest.raises(TypeError, match="not supported"):
        simulate_monolithic(object(), mode="state_vector", max_bond_dimension=1)


def test_mps_mode_rejects_unknown_option():
    with pytest.raises(TypeError, match="Unsupported MPS option"):
        simulate_monolithic(object(), mode="mps", unknown_option=True)


def test_mps_mode_accepts_supported_options_before_circuit_decoding():
    with pytest.raises(AttributeError, match="model_dump_json"):
        simulate_monolithic(object(), mode="mps", max_bond_dimension=1, truncation_threshold=1e-14)


def test_mps_mode_accepts_none_bond_dimension_before_circuit_decoding():
    with pytest.raises(AttributeError, match="model_dump_json"):
        simulate_monolithic(object(), mode="mps", max_bond_dimension=None)


def test_mps_mode_rejects_zero_bond_dimension():
    with pytest.raises(ValueError, match="max_bond_dimension"):
        simulate_monolithic(object(), mode="mps", max_bond_dimension=0)


@pytest.mark.parametrize("threshold", [-1.0, float("nan"), float("inf")])
def test_mps_mode_rejects_invalid_truncation_threshold(threshold):
    with pytest.raises(ValueError, match="truncation_threshold"):
        simulate_monolithic(object(), mode="mps", truncation_threshold=threshold)


def test_invalid_distributed_mode_raises_before_decoding_circuit():
    with pytest.raises(ValueError, match="Unsupported distributed simulation mode"):
        simulate_distributed(object(), mode="state_vector")


def test_stabilizer_statevector_extraction_is_rejected():
    with pytest.raises(NotImplementedError, match="simulate_monolithic_shots"):
        simulate_monolithic(object(), mode="stabilizer")


def test_shots_mode_parsing_precedes_decoding():
    with pytest.raises(AttributeError, match="model_dump_json"):
        simulate_monolithic_shots(object(), mode="sv")


# ---- JSON decoding (serde semantics of src/types.rs) ----------------------------------------


def test_num_qubits_is_max_base_plus_size():
    c = decode_circuit_json(json.dumps({
        "qregs": {"a": {"name": "a", "size": 3, "base": 0}, "b": {"name": "b", "size": 2, "base": 5}},
        "instructions": []}))
    assert c.num_qubits() == 7 and c.num_cbits() == 0


def test_no_registers_means_zero_qubits():
    c = decode_circuit_json(json.dumps({"qregs": {}, "instructions": []}))
    assert c.num_qubits() == 0


def test_extra_fields_are_ignored_and_ints_accepted_as_floats():
    c = decode_circuit_json(json.dumps({
        "qregs": {"q": {"name": "q", "size": 1, "base": 0, "extra": 1}},
        "instructions": [{"kind": "rx", "qubit": 0, "theta": 1, "qubits": [0], "params": [1.0],
                          "label": "x"}],
        "metadata": {"anything": True}}))
    assert c.instructions[0].fields["theta"] == 1.0


@pytest.mark.parametrize("bad", [
    {"instructions": []},                                              # missing qregs
    {"qregs": {}},                                                     # missing instructions
    {"qregs": {}, "cregs": None, "instructions": []},                  # null map
    {"qregs": {}, "instructions": [{"kind": "nope", "qubit": 0}]},     # unknown variant
    {"qregs": {}, "instructions": [{"kind": "rx", "qubit": 0}]},       # missing field
    {"qregs": {}, "instructions": [{"kind": "x", "qubit": 1.0}]},      # float for usize
    {"qregs": {}, "instructions": [{"kind": "x", "qubit": -1}]},       # negative usize
    {"qregs": {}, "instructions": [{"kind": "x", "qubit": True}]},     # bool for usize
    {"qregs": {}, "instructions": [{"kind": "rx", "qubit": 0, "theta": "1"}]},
    {"qregs": {}, "instructions": [{"qubit": 0}]},                     # no tag
    {"qregs": {"q": {"name": "q", "size": 1}}, "instructions": []},    # register field
    {"qregs": {}, "instructions": [{"kind": "gate", "name": "remote_cx", "qubits": [0, 1]}]},
])
def test_decode_rejects_what_serde_rejects(bad):
    with pytest.raises(CircuitDecodeError):
        decode_circuit_json(json.dumps(bad))


def test_invalid_json_text_rejected():
    with pytest.raises(CircuitDecodeError):
        decode_circuit_json("{not json")
    with pytest.raises(CircuitDecodeError):
        decode_circuit_json('{"qregs": {}, "instructions": [{"kind": "rx", "qubit": 0, "theta": NaN}]}')


def test_encode_fields_in_reference_order():
    c = JsonCircuit(5, [g("cu", 1, 3, 0.1, 0.2, 0.3, 0.4), g("cswap", 4, 0, 2),
                        g("rz", 2, 0.7), g("measure", 3, 6),
                        cond(1, 2, 3, cond(4, 1, 1, g("cp", 0, 1, 0.5))),
                        gate("Remote_Link_PSI_minus", [3, 4]), gate("circuit-7", [0]),
                        gate("foo", [1]), {"kind": "barrier"}, {"kind": "classical", "name": "c"}],
                    ncbits=2)
    p = encode(decode_circuit_json(c.model_dump_json()))
    k = nat.KIND
    r = p.insts
    assert r[0]["kind"] == k["cu"] and r[0]["q"][:2].tolist() == [1, 3]
    assert r[0]["p"].tolist() == [0.1, 0.2, 0.3, 0.4]
    assert r[1]["kind"] == k["cswap"] and r[1]["q"][:3].tolist() == [4, 0, 2]
    assert r[2]["kind"] == k["rz"] and r[2]["p"][0] == 0.7
    assert r[3]["kind"] == k["measure"] and r[3]["cbit"] == 6 and r[3]["nq"] == 1
    assert r[4]["kind"] == k["cp"] and r[4]["cond_count"] == 2
    assert p.conds.tolist() == [(1, 2, 3), (4, 1, 1)]
    assert r[5]["kind"] == k["g_psi_minus"] and r[5]["nq"] == 2
    assert r[6]["kind"] == k["g_opaque"] and r[7]["kind"] == k["g_unsupported"]
    assert p.gate_names[7] == "foo"
    assert r[8]["kind"] == k["barrier"] and r[9]["kind"] == k["classical"]
    assert p.num_cbits == 2 and p.cbit_space == 7


def test_generic_remote_gate_needs_two_qubits():
    c = JsonCircuit(3, [gate("nonlocal_cz", [0, 1, 2])])
    with pytest.raises(ValueError):
        encode(decode_circuit_json(c.model_dump_json()))


def test_format_cbits_msb_first_unwritten_zero():
    bits = np.array([1, -1, 0, 1], dtype=np.int32)
    assert format_cbits(bits, 4) == "1001"
    assert format_cbits(bits, 0) == ""
    assert format_cbits(bits, 3) == "001"


def test_inst_record_layout_matches_header():
    hdr = (ROOT / "include" / "dqsim_cuda.h").read_text()
    assert "int32_t q[DQ_MAX_INST_QUBITS]" in hdr
    assert nat.INST_DTYPE.fields["cbit"][1] == 40
    assert nat.INST_DTYPE.fields["p"][1] == 48
    assert nat.INST_DTYPE.fields["cond_first"][1] == 80
    kinds = re.search(r"enum dq_kind \{(.*?)\};", hdr, re.S).group(1)
    kinds = re.sub(r"/\*.*?\*/", "", kinds, flags=re.S)
    names = re.findall(r"\bDQ_([A-Z0-9_]+)", kinds)
    names = [n for n in names if n != "KIND_COUNT"]
    assert len(names) == len(nat.KIND_NAMES)


# ---- the C ABI library -------------------------------------------------------------------------


def test_library_exports_every_declared_symbol(engine_lib):
    hdr = (ROOT / "include" / "dqsim_cuda.h").read_text()
    declared = re.findall(r"^DQ_API\s+[\w\s\*]+?\b(dq_\w+)\s*\(", hdr, re.M)
    assert len(declared) >= 25
    lib = ctypes.CDLL(str(nat.LIB_PATH))
    for name in declared:
        assert hasattr(lib, name), f"{name} declared but not exported"
    assert engine_lib.dq_abi_version() == 1


def test_binding_signatures_cover_the_header(engine_lib):
    hdr = (ROOT / "include" / "dqsim_cuda.h").read_text()
    declared = set(re.findall(r"^DQ_API\s+[\w\s\*]+?\b(dq_\w+)\s*\(", hdr, re.M))
    bound = {name for name, _, _ in nat.SIGNATURES}
    assert declared == bound


def test_null_handle_and_bad_args_return_status(engine_lib):
    assert engine_lib.dq_state_destroy(None) == 0
    n = ctypes.c_uint32(0)
    assert engine_lib.dq_state_num_qubits(None, ctypes.byref(n)) == nat.DQ_ERR_INVALID_ARG
    assert "null" in nat.last_error()
    assert engine_lib.dq_rng_f64(1, 0, 4, None) == nat.DQ_ERR_INVALID_ARG
    blk = np.zeros(16, dtype=np.uint32)
    assert engine_lib.dq_chacha_block(blk.ctypes.data, 7, blk.ctypes.data) == nat.DQ_ERR_INVALID_ARG


def test_mps_entry_points_reject_bad_arguments_without_a_gpu(engine_lib):
    L = engine_lib
    assert L.dq_mps_destroy(None) == 0
    h = ctypes.c_void_p()
    assert L.dq_mps_create(0, 0, 0, 1e-12, ctypes.byref(h)) == nat.DQ_ERR_INVALID_ARG
    assert "qubit count" in nat.last_error()
    # any threshold is accepted (MpsSimulator::new takes any f64): without a GPU the
    # call gets as far as the device check
    assert L.dq_mps_create(4, 0, 0, -1.0, ctypes.byref(h)) in (nat.DQ_ERR_NO_DEVICE, nat.DQ_ERR_CUDA)
    assert L.dq_mps_create(4, 0, 0, 1e-12, None) == nat.DQ_ERR_INVALID_ARG
    st = nat.MpsStats()
    assert L.dq_mps_run(None, None, 0, None, 0, 0, None, 0, ctypes.byref(st)) == nat.DQ_ERR_INVALID_ARG
    assert L.dq_mps_bond_dims(None, None) == nat.DQ_ERR_INVALID_ARG
    assert L.dq_mps_apply_2q(None, 0, 1, None) == nat.DQ_ERR_INVALID_ARG
    # an unconditional gate on three qubits is rejected while lowering, before any device work
    from dqsim_bosonic_b200.circuit import decode_circuit_json, encode
    from _circuits import JsonCircuit, g
    p = encode(decode_circuit_json(JsonCircuit(3, [g("h", 0), g("ccx", 0, 1, 2)]).model_dump_json()))
    rc = L.dq_mps_run_shots(0, 3, 0, 1e-12, nat.ptr(p.insts), p.ninst, None, 0, 1, 0, 4, None, 0, 0,
                            ctypes.byref(st))
    assert rc == nat.DQ_ERR_UNSUPPORTED and st.failed_inst == 1
