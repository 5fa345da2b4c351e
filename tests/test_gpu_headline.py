"""Parity at the benchmark's own sizes (needs a B200; ~40 GB of HBM).

The bench times ``StatevectorSimulator(exec="fused").simulate`` of the
30-qubit QFT (x on a seeded half of the qubits, then the QFT with its swap
network) and of the two-node distributed variant (2 x 14 data + 2 link
qubits, remote_link_psi_minus + nonlocal_cz).  These tests check exactly
those runs:

* the fused QFT30 state against the closed form of the QFT of a basis state,
  amp[w] = exp(2 pi i rev(x) rev(w) / 2^30) / 2^15 (rev = 30-bit reversal;
  src/gates.rs:135 cp = controlled p, the circuit applies h(j) then
  cp(pi/2^(k-j)) controlled by k > j, then swap(j, 29-j)), on 2^20 random
  indices and a contiguous block, plus the norm of the whole state;
* the fused QFT30 and distributed states against the exact per-gate engine
  (bit-identical to the oracle, tests/test_gpu_parity.py) over all 2^30
  amplitudes, within the 1e-12 amplitude tolerance.
"""
import math

import numpy as np
import pytest

from _circuits import distributed_qft_variant, qft_with_x

pytestmark = pytest.mark.gpu

ATOL = 1e-12
N = 30


class _CudaArray:
    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


def device_view(res):
    """The result's state as a complex128 CUDA tensor (canonical layout)."""
    import torch

    st = res.state_handle
    ptr, _ = st.device_ptr()
    flat = torch.as_tensor(_CudaArray(ptr, 2 << st.n), device=torch.device("cuda", st.device))
    return torch.view_as_complex(flat.view(-1, 2))


def bit_reverse(t, n):
    import torch

    out = torch.zeros_like(t)
    for b in range(n):
        out |= ((t >> b) & 1) << (n - 1 - b)
    return out


def chunked_norm(v, chunk=1 << 26):
    tot = 0.0
    for s in range(0, v.numel(), chunk):
        c = v[s:s + chunk]
        tot += float((c.real * c.real + c.imag * c.imag).sum())
    return tot


def chunked_max_diff(a, b, chunk=1 << 26):
    m = 0.0
    for s in range(0, a.numel(), chunk):
        m = max(m, float((a[s:s + chunk] - b[s:s + chunk]).abs().max()))
    return m


def x_mask_of(circ):
    mask = 0
    for ins in circ.instructions:
        if ins["kind"] == "x":
            mask ^= 1 << ins["qubit"]
    return mask


def test_qft30_fused_matches_closed_form(gpu):
    import torch

    from dqsim_bosonic_b200 import StatevectorSimulator

    circ = qft_with_x(N, 1234)
    x = x_mask_of(circ)
    assert x != 0
    res = StatevectorSimulator(seed=7, device=0, exec="fused").simulate(circ)
    v = device_view(res)
    dev = v.device
    assert abs(chunked_norm(v) - 1.0) < 1e-10
    g = torch.Generator(device=dev)
    g.manual_seed(1234)
    w = torch.randint(0, 1 << N, (1 << 20,), device=dev, dtype=torch.int64, generator=g)
    w = torch.cat([w, torch.arange(0, 1 << 16, device=dev, dtype=torch.int64),
                   torch.tensor([(1 << N) - 1, 1 << (N - 1), x], device=dev, dtype=torch.int64)])
    rx = int(format(x, f"0{N}b")[::-1], 2)
    k = (rx * bit_reverse(w, N)) & ((1 << N) - 1)
    ph = (2.0 * math.pi / (1 << N)) * k.to(torch.float64)
    want = torch.complex(torch.cos(ph), torch.sin(ph)) / float(1 << (N // 2))
    err = float((v[w] - want).abs().max())
    assert err <= ATOL, err
    del v
    res.state_handle.release()
    torch.cuda.synchronize()


@pytest.mark.parametrize("which", ["qft30", "distributed30"])
def test_fused_matches_exact_engine_at_30_qubits(gpu, which):
    import torch

    from dqsim_bosonic_b200 import StatevectorSimulator

    circ = qft_with_x(N, 1234) if which == "qft30" else distributed_qft_variant(14, 1234)
    a = StatevectorSimulator(seed=7, device=0, exec="fused").simulate(circ)
    b = StatevectorSimulator(seed=7, device=0, exec="per_gate").simulate(circ)
    assert a.num_qubits == N and b.num_qubits == N
    va, vb = device_view(a), device_view(b)
    err = chunked_max_diff(va, vb)
    assert err <= ATOL, (which, err)
    assert abs(chunked_norm(va) - 1.0) < 1e-10
    # the marginal the bench reads agrees too
    top = list(range(N - 1, N - 11, -1))
    pa, pb = a.probability_array(top), b.probability_array(top)
    assert np.max(np.abs(pa - pb)) < 1e-12
    del va, vb
    a.state_handle.release()
    b.state_handle.release()
    torch.cuda.synchronize()
