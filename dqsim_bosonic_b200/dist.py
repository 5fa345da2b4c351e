"""Sharding of independent work across ranks (one process per GPU).

Shot trajectories and parameter sets are independent, so they shard with no
exchange on the data path: rank ``r`` of ``w`` takes a contiguous slice, keeps
the global indices (shot ``i`` still draws from ``base_seed + i``, so the
result does not depend on the number of ranks), and one collective at the end
merges the results:

* counts: a dense histogram over the ``2^ncbits`` classical outcomes summed
  with ``all_reduce`` (``ncbits <= 24``), otherwise the per-rank dicts are
  gathered with ``all_gather_object``;
* per-set values (energies, gradients): ``all_gather`` of equal-sized padded
  slices, trimmed to the global batch.

The process group is the caller's (``torch.distributed``; NCCL on GPUs, gloo
for CPU tests).  Nothing here touches device memory of another rank.
"""
from __future__ import annotations

import numpy as np

MAX_DENSE_CBITS = 24


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) slice of ``total`` items for ``rank`` of ``world``;
    the first ``total % world`` ranks take one extra item."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    if total < 0:
        raise ValueError("total must be >= 0")
    base, extra = divmod(total, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def counts_to_hist(counts: dict[str, int], ncbits: int) -> np.ndarray:
    h = np.zeros(1 << ncbits, dtype=np.int64)
    for k, v in counts.items():
        h[int(k, 2) if k else 0] += v
    return h


def hist_to_counts(h: np.ndarray, ncbits: int) -> dict[str, int]:
    out = {}
    for i in np.nonzero(h)[0].tolist():
        out[format(i, f"0{ncbits}b") if ncbits else ""] = int(h[i])
    return out


def merge_counts(counts: dict[str, int], ncbits: int, group=None) -> dict[str, int]:
    """Sum per-rank counts over the process group (identity without one)."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return dict(counts)
    if ncbits <= MAX_DENSE_CBITS:
        dev = _collective_device(group)
        h = torch.from_numpy(counts_to_hist(counts, ncbits)).to(dev)
        dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
        return hist_to_counts(h.cpu().numpy(), ncbits)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, dict(counts), group=group)
    out: dict[str, int] = {}
    for p in parts:
        for k, v in p.items():
            out[k] = out.get(k, 0) + v
    return out


def gather_rows(local: np.ndarray, total: int, group=None) -> np.ndarray:
    """Concatenate the ranks' contiguous slices (shard_range order) of a
    per-item array into the global ``total`` rows."""
    import torch
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return np.asarray(local)
    world = dist.get_world_size(group)
    per = -(-total // world)
    a = np.asarray(local, dtype=np.float64)
    pad = np.zeros((per,) + a.shape[1:], dtype=np.float64)
    pad[: a.shape[0]] = a
    dev = _collective_device(group)
    t = torch.from_numpy(pad).to(dev)
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    rows = []
    for r in range(world):
        lo, hi = shard_range(total, r, world)
        rows.append(outs[r][: hi - lo].cpu().numpy())
    return np.concatenate(rows, axis=0)


def _collective_device(group=None):
    import torch
    import torch.distributed as dist

    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def simulate_shots_sharded(sim, circuit, shots: int, group=None) -> dict[str, int]:
    """``simulate_shots`` with the shots split across the process group; every
    rank returns the merged counts (identical to a single-rank run).  ``sim``
    is a ``StatevectorSimulator`` or an ``MpsSimulator``."""
    import torch.distributed as dist

    from .batch import run_trajectories
    from .circuit import format_cbits
    from .mps import MpsSimulator, run_mps_shots
    from .statevector import _entropy_u64, _parse

    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    prog, _ = _parse(circuit)
    base_seed = sim._seed if sim._seed is not None else _entropy_u64()
    lo, hi = shard_range(shots, rank, world)
    counts: dict[str, int] = {}
    if hi > lo:
        seed0 = (base_seed + lo) & ((1 << 64) - 1)
        if isinstance(sim, MpsSimulator):  # MPS shots (mps/simulator.rs:368-385), same seeding
            bits, _ = run_mps_shots(prog, seed0, hi - lo, sim.device, sim._max_bond, sim._threshold)
        else:
            bits, _, _ = run_trajectories(prog, seed0, hi - lo, sim.device)
        for row in bits:
            k = format_cbits(row, prog.num_cbits)
            counts[k] = counts.get(k, 0) + 1
    return merge_counts(counts, prog.num_cbits, group)
