"""The allocation-free p1 entry point (needs a B200).

dq_measure_p1_noalloc serves callers that cannot allocate device memory:
hosts with a fixed device-memory budget, embedders whose allocator must not
be bypassed, code running where cudaMalloc is not permitted.  The test acts as
such a caller: it owns the state and the output buffer, calls the entry
point through the C ABI twice in a row (the shared static scratch keeps the
previous call's contents), and compares both results with dq_measure_p1.
This file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

from dqsim_bosonic_b200 import _native as nat

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def test_p1_noalloc_matches_measure_p1(gpu):
    import torch

    n = 18
    rng = np.random.default_rng(11)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    v /= np.linalg.norm(v)
    st = nat.State(n, 0)
    st.upload(v)
    amps, _ = st.device_ptr()
    torch.cuda.set_device(0)
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    L = nat.lib()
    for qubit in (0, 7, n - 1):
        want = ctypes.c_double(0.0)
        nat.check(L.dq_measure_p1(st.handle, qubit, ctypes.byref(want)), "dq_measure_p1")
        for call in range(2):  # two calls in a row share the static scratch
            out.zero_()
            torch.cuda.synchronize()
            rc = L.dq_measure_p1_noalloc(amps, n, qubit, out.data_ptr() + 8 * call, None)
            nat.check(rc, "dq_measure_p1_noalloc")
            torch.cuda.synchronize()
            got = out[call].item()
            assert abs(got - want.value) <= RTOL * abs(want.value), (qubit, call, got, want.value)
    # the host-side reference value agrees too
    assert abs(out[1].item() - float(np.sum(np.abs(v[1 << (n - 1):]) ** 2))) < 1e-12


def test_p1_noalloc_rejects_bad_sizes(gpu):
    import torch

    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    src = torch.zeros(4, dtype=torch.float64, device="cuda:0")
    L = nat.lib()
    assert L.dq_measure_p1_noalloc(src.data_ptr(), 35, 0, out.data_ptr(), None) == nat.DQ_ERR_INVALID_ARG
    assert "1..34" in nat.last_error()
    assert L.dq_measure_p1_noalloc(src.data_ptr(), 1, 1, out.data_ptr(), None) == nat.DQ_ERR_INVALID_ARG
    assert L.dq_measure_p1_noalloc(None, 1, 0, out.data_ptr(), None) == nat.DQ_ERR_INVALID_ARG
