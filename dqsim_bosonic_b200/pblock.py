"""Block states of the p-block simulator and their merge on the GPU.

The reference's p-block simulator keeps one state vector per group of qubits
that have interacted (``Block``, src/distributed/pblock/model.rs:7-27) and
merges two groups into the tensor product of their states when a gate spans
them (``merge_blocks``, model.rs:35-57).  Here a block's state lives in HBM
(an engine state) and the merge is one kernel (``dq_block_merge``) that
writes the merged state; gates on a block run through the engine like on any
state (``Block.state``).
"""
from __future__ import annotations

import numpy as np

from . import _native as nat

__all__ = ["Block", "merge_blocks"]


class Block:
    """The state of a group of qubits: ``qubits`` ascending and distinct
    (the constructor sorts and removes duplicates, as ``Block::new`` does),
    bit k of the state index is ``qubits[k]``; it starts in |0...0>."""

    def __init__(self, qubits, device: int = 0, *, _state: nat.State | None = None):
        self.qubits = sorted(set(int(q) for q in qubits))
        self.device = int(device)
        self.state = _state if _state is not None else nat.State(len(self.qubits), self.device)

    def local(self, phys: int) -> int:
        """Index of physical qubit ``phys`` in this block."""
        try:
            return self.qubits.index(int(phys))
        except ValueError:
            raise ValueError(f"qubit {phys} not in block {self.qubits}") from None

    def statevector(self) -> np.ndarray:
        return self.state.download()

    def release(self) -> None:
        self.state.release()


def merge_blocks(a: Block, b: Block) -> Block:
    """The tensor product of ``a`` and ``b`` as one block over the ascending
    union of their qubits (bit-identical to the reference's merge).  The
    inputs are left as they are; release them when they are no longer used."""
    if a.device != b.device:
        raise ValueError("blocks must live on one device")
    qubits = sorted(set(a.qubits) | set(b.qubits))
    out = nat.State(len(qubits), a.device)
    qa = np.asarray(a.qubits, dtype=np.uint32)
    qb = np.asarray(b.qubits, dtype=np.uint32)
    nat.check(nat.lib().dq_block_merge(a.state.handle, nat.ptr(qa) if qa.size else None, qa.size,
                                       b.state.handle, nat.ptr(qb) if qb.size else None, qb.size,
                                       out.handle), "dq_block_merge")
    return Block(qubits, a.device, _state=out)
