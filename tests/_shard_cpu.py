"""CPU shard backend for the sharded-state orchestration tests: a numpy shard
whose gates run through the oracle (test infrastructure only)."""
import numpy as np

import _oracle as orc


class CpuShard:
    def __init__(self, nl: int, rank: int = 0):
        self.nl = nl
        self.state = np.zeros(1 << nl, dtype=np.complex128)
        self.state[0] = 1.0

    def run(self, insts):
        self.state[:] = orc.run_unitary(insts, self.nl, init=self.state)

    def p1(self, a):
        return orc.p1(self.state, a)

    def collapse(self, a, outcome, p1):
        if outcome == 1:
            norm = max(np.sqrt(p1), 1e-15)
        else:
            norm = max(np.sqrt(max(1.0 - p1, 0.0)), 1e-15)
        idx = np.arange(self.state.size)
        keep = ((idx >> a) & 1) == outcome
        self.state[~keep] = 0.0
        self.state[keep] = self.state[keep] / norm

    def marginal(self, positions):
        return orc.marginal(self.state, positions)

    def view(self):
        import torch

        return torch.from_numpy(self.state.view(np.float64))

    def zero(self):
        self.state[:] = 0.0

    def download(self):
        return self.state.copy()

    def release(self):
        pass
