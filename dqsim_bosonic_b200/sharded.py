"""One statevector sharded over 2^g ranks by its top g physical qubits.

A state of n qubits is too large for one GPU from 34 qubits on (2^34 x 16 B =
256 GiB).  Here rank r of 2^g holds the 2^(n-g) amplitudes whose physical
index has r in its top g bits: physical positions 0 .. n_l - 1 are "local"
(n_l = n - g), positions n_l .. n - 1 are "global" (the rank's bits).

Logical qubits map to physical positions through a relabelling the run keeps,
and every global position j carries a flip bit (the logical value of the
qubit there is rank bit j XOR flip j):
  * swap gates are relabellings and x on a global qubit is a flip: no data
    moves;
  * a gate whose qubits are all local runs on the shard through the engine
    (consecutive ones batched into one fused ``dq_run``);
  * a gate touching a global qubit is reduced per rank where its matrix
    allows: a global control either drops the gate (control bit 0) or is
    removed from it (cx -> x, ccx -> cx, cp -> p, cu -> u3 and a phase ...),
    and a diagonal gate on a global qubit becomes a phase on the shard or a
    smaller diagonal on the local qubits (z, s, t, p, rz on a global target;
    cz, cp, crz, rzz with a global member);
  * anything else (a global target of a non-diagonal gate, a measured global
    qubit) first exchanges the global qubit with a local one.

The exchange of global position j with local position a is the one data-path
collective: partner ranks r and r ^ 2^j swap the part of their shards whose
local bit a differs from their rank bit j, 2^(n_l - 1) amplitudes on each
side (blocks of 2^a contiguous amplitudes; the victim is taken from the top
local positions so the blocks stay large), in place through a chunk buffer.
Measurement sums the ranks' partial p1 with one all-reduce and every rank
draws the outcome from the same ChaCha8 stream
(``simulate`` semantics: one f64 per measure / reset, in program order), so
outcomes, classical bits and the collapse match a single-state run except
where |r - p1| is at rounding level (counted in ``boundary_draws``).

Ranks are either one process per GPU (``torch.distributed``: NCCL point to
point on CUDA tensors, gloo on CPU) or several shards held by one process
(``LocalShards``), which runs every rank's step in turn and exchanges by
copies: the same orchestration with no collective library, for one-GPU runs
and tests.  The per-shard engine is a backend object (``NativeShard``: an
engine state on a GPU).
"""
from __future__ import annotations

import ctypes
import math
from typing import Any, Sequence

import numpy as np

from . import _native as nat
from .circuit import Program

K = nat.KIND
_U64 = (1 << 64) - 1

# ---- gate tables ------------------------------------------------------------------------

# leading control qubits of the controlled kinds, and the kind left when one
# control is dropped (the kept controls stay in front, in order)
_NCTL = {
    K["cx"]: 1, K["cy"]: 1, K["cz"]: 1, K["ch"]: 1, K["csx"]: 1, K["crx"]: 1, K["cry"]: 1,
    K["crz"]: 1, K["cu1"]: 1, K["cp"]: 1, K["cu3"]: 1, K["cu"]: 1, K["ccx"]: 2, K["c3x"]: 3,
    K["c4x"]: 4, K["cswap"]: 1, K["g_cx"]: 1, K["g_cz"]: 1,
}
_DROP = {
    K["cx"]: K["x"], K["cy"]: K["y"], K["cz"]: K["z"], K["ch"]: K["h"], K["csx"]: K["sx"],
    K["crx"]: K["rx"], K["cry"]: K["ry"], K["crz"]: K["rz"], K["cu1"]: K["u1"], K["cp"]: K["p"],
    K["cu3"]: K["u3"], K["cu"]: K["u3"], K["ccx"]: K["cx"], K["c3x"]: K["ccx"], K["c4x"]: K["c3x"],
    K["cswap"]: K["swap"], K["g_cx"]: K["x"], K["g_cz"]: K["z"],
}
# diagonal two-qubit kinds symmetric in their qubits (a global "target" can
# act as the control)
_SYM_DIAG = {K["cz"], K["cp"], K["cu1"], K["g_cz"]}
_NOOP = {K["id"], K["u0"], K["barrier"], K["classical"], K["g_noop"]}
_ONE_Q = {K[k] for k in ("id", "x", "y", "z", "h", "s", "sdg", "t", "tdg", "sx", "sxdg", "u3", "u2",
                         "u1", "u", "p", "rx", "ry", "rz", "u0")}


def _phase_1q(kind: int, p: np.ndarray, e: int) -> complex | None:
    """The phase a diagonal one-qubit kind puts on basis value e, or None if
    the kind is not diagonal."""
    if kind in (K["id"], K["u0"]):
        return 1.0
    if kind == K["z"]:
        return -1.0 if e else 1.0
    if kind == K["s"]:
        return 1j if e else 1.0
    if kind == K["sdg"]:
        return -1j if e else 1.0
    if kind == K["t"]:
        return complex(math.cos(math.pi / 4), math.sin(math.pi / 4)) if e else 1.0
    if kind == K["tdg"]:
        return complex(math.cos(math.pi / 4), -math.sin(math.pi / 4)) if e else 1.0
    if kind in (K["p"], K["u1"]):
        return complex(math.cos(p[0]), math.sin(p[0])) if e else 1.0
    if kind == K["rz"]:
        h = 0.5 * p[0]
        return complex(math.cos(h), math.sin(h) if e else -math.sin(h))
    return None


def _inst(kind: int, qubits: Sequence[int], params: Sequence[float] = ()) -> np.ndarray:
    r = np.zeros((), dtype=nat.INST_DTYPE)
    r["kind"] = kind
    r["nq"] = len(qubits)
    r["q"][:] = -1
    for i, q in enumerate(qubits):
        r["q"][i] = q
    for i, v in enumerate(params):
        r["p"][i] = v
    return r


def _phase_insts(phase: complex, q: int) -> list[np.ndarray]:
    """exp(i g) on every amplitude as two diagonal gates on physical qubit q:
    p(2g) rz(-2g) = exp(i g) I."""
    if phase == 1.0:
        return []
    g = math.atan2(phase.imag, phase.real)
    return [_inst(K["p"], [q], [2.0 * g]), _inst(K["rz"], [q], [-2.0 * g])]


# ---- communication ----------------------------------------------------------------------

class _DistComm:
    """One rank per process over a torch.distributed group."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.local_ranks = [self.rank]

    def _device(self):
        import torch

        if self.dist.get_backend(self.group) == "nccl":
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def allreduce(self, parts: list[np.ndarray]) -> np.ndarray:
        import torch

        t = torch.from_numpy(np.ascontiguousarray(parts[0], dtype=np.float64)).to(self._device())
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def swap_regions(self, views: dict, pairs_for, chunk: int) -> None:
        """views[rank] -> flat float64 tensor; pairs_for(rank) -> (partner,
        [(start, length)] in float64 units): the k-th range of a rank is sent
        to and received from the partner's k-th range (same lengths)."""
        import torch

        (r,) = self.local_ranks
        v = views[r]
        partner, ranges = pairs_for(r)
        gr = self.dist.get_global_rank(self.group, partner) if self.group is not None else partner
        tmp = torch.empty(min(chunk, max((l for _, l in ranges), default=1)), dtype=v.dtype,
                          device=v.device)
        for start, length in ranges:
            for off in range(0, length, chunk):
                m = min(chunk, length - off)
                src = v[start + off: start + off + m]
                dst = tmp[:m]
                reqs = [self.dist.isend(src, gr, group=self.group),
                        self.dist.irecv(dst, gr, group=self.group)]
                for q in reqs:
                    q.wait()
                src.copy_(dst)
        if v.is_cuda:
            torch.cuda.synchronize(v.device)


class LocalShards:
    """All 2^g ranks in one process (every step runs for each shard in turn;
    exchanges are copies between the shards' memory)."""

    def __init__(self, world: int):
        self.rank = 0
        self.world = int(world)
        self.local_ranks = list(range(self.world))

    def allreduce(self, parts: list[np.ndarray]) -> np.ndarray:
        out = np.zeros_like(np.asarray(parts[0], dtype=np.float64))
        for p in parts:
            out = out + p
        return out

    def swap_regions(self, views: dict, pairs_for, chunk: int) -> None:
        import torch

        done = set()
        for r in self.local_ranks:
            partner, ranges = pairs_for(r)
            if (partner, r) in done:
                continue
            done.add((r, partner))
            a, b = views[r], views[partner]
            _, pranges = pairs_for(partner)
            for (start, length), (pstart, _) in zip(ranges, pranges):
                for off in range(0, length, chunk):
                    m = min(chunk, length - off)
                    x = a[start + off: start + off + m]
                    y = b[pstart + off: pstart + off + m]
                    t = x.clone()
                    x.copy_(y)
                    y.copy_(t)
        for r in self.local_ranks:
            if views[r].is_cuda:
                torch.cuda.synchronize(views[r].device)


# ---- the GPU shard backend --------------------------------------------------------------

class _CudaArray:
    def __init__(self, ptr: int, count: int):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


class NativeShard:
    """A shard on one GPU: an engine state of n_l qubits."""

    def __init__(self, nl: int, device: int, exec_mode: int = nat.EXEC_FUSED):
        self.nl = nl
        self.device = device
        self.exec_mode = exec_mode
        self.state = nat.State(nl, device)

    def run(self, insts: np.ndarray) -> None:
        from .statevector import run_program

        prog = Program(insts, np.zeros(0, dtype=nat.COND_DTYPE), self.nl, 0, 1, {})
        run_program(self.state, prog, 0, nat.SEM_SIMULATE, self.exec_mode)

    def p1(self, a: int) -> float:
        out = ctypes.c_double()
        nat.check(nat.lib().dq_measure_p1(self.state.handle, a, ctypes.byref(out)), "dq_measure_p1")
        return out.value

    def collapse(self, a: int, outcome: int, p1: float) -> None:
        nat.check(nat.lib().dq_collapse(self.state.handle, a, outcome, p1), "dq_collapse")

    def marginal(self, positions: Sequence[int]) -> np.ndarray:
        q = np.asarray(positions, dtype=np.uint32)
        out = np.empty(1 << len(q), dtype=np.float64)
        nat.check(nat.lib().dq_marginal_probs(self.state.handle, nat.ptr(q), len(q), nat.ptr(out)),
                  "dq_marginal_probs")
        return out

    def view(self):
        """The shard as a flat float64 CUDA tensor (re, im interleaved); the
        engine's stream is drained first and torch's work is drained by the
        caller before the engine runs again."""
        import torch

        ptr, _ = self.state.device_ptr()
        return torch.as_tensor(_CudaArray(ptr, 2 << self.nl), device=torch.device("cuda", self.device))

    def zero(self) -> None:
        import torch

        self.view().zero_()
        torch.cuda.synchronize(self.device)

    def download(self) -> np.ndarray:
        return self.state.download()

    def release(self) -> None:
        self.state.release()


# ---- the sharded state ------------------------------------------------------------------

class ShardedStatevector:
    """``n`` logical qubits over ``comm.world`` = 2^g ranks.

    ``comm``: ``None`` for the initialised default torch.distributed group, a
    process group, or a ``LocalShards``.  ``backend(nl, rank)`` makes a rank's
    shard (default: ``NativeShard`` on ``device``).  The state starts in
    |0...0>.  ``chunk``: exchange message size in amplitudes."""

    def __init__(self, n: int, comm: Any = None, *, device: int = 0, backend=None,
                 exec: str = "fused", chunk: int = 1 << 22):
        if isinstance(comm, LocalShards):
            self.comm = comm
        else:
            self.comm = _DistComm(comm)
        W = self.comm.world
        g = W.bit_length() - 1
        if W < 1 or (1 << g) != W:
            raise ValueError("the number of ranks must be a power of two")
        if n - g < 1:
            raise ValueError(f"{n} qubits cannot be sharded over {W} ranks")
        self.n, self.g, self.nl = int(n), g, int(n) - g
        self.chunk = int(chunk)
        self.pos = list(range(n))   # logical qubit -> physical position
        self.at = list(range(n))    # physical position -> logical qubit
        self.flip = [0] * g         # per global position
        self.boundary_draws = 0
        self.exchanges = 0
        em = nat.EXEC_FUSED if exec == "fused" else nat.EXEC_PER_GATE
        if backend is None:
            def backend(nl, rank):
                return NativeShard(nl, device, em)
        self.shards = {r: backend(self.nl, r) for r in self.comm.local_ranks}
        for r, s in self.shards.items():
            if r != 0:
                s.zero()
        self._pending = {r: [] for r in self.comm.local_ranks}

    # -- layout helpers --
    def _gbit(self, rank: int, q: int) -> int:
        """Logical value of global qubit q on ``rank``."""
        j = self.pos[q] - self.nl
        return ((rank >> j) & 1) ^ self.flip[j]

    def _is_global(self, q: int) -> bool:
        return self.pos[q] >= self.nl

    def _emit(self, rank: int, inst: np.ndarray) -> None:
        self._pending[rank].append(inst)

    def _flush(self) -> None:
        for r, lst in self._pending.items():
            if lst:
                self.shards[r].run(np.array(lst, dtype=nat.INST_DTYPE))
                lst.clear()

    def _make_local(self, qubits: Sequence[int], keep: Sequence[int]) -> None:
        """Exchange each global qubit of ``qubits`` with a local position whose
        qubit is not in ``keep`` (highest positions first)."""
        for q in qubits:
            if not self._is_global(q):
                continue
            a = next((p for p in range(self.nl - 1, -1, -1) if self.at[p] not in keep), None)
            if a is None:
                raise ValueError("not enough local qubits for this gate on the sharded state")
            self._exchange(self.pos[q] - self.nl, a)

    def _exchange(self, j: int, a: int) -> None:
        self._flush()
        views = {r: s.view() for r, s in self.shards.items()}
        nl = self.nl

        def pairs_for(r):
            v = 1 - ((r >> j) & 1)        # the local bit a of the amplitudes that move
            blk = 1 << a
            ranges = [(2 * (k * 2 * blk + v * blk), 2 * blk) for k in range(1 << (nl - 1 - a))]
            return r ^ (1 << j), ranges

        self.comm.swap_regions(views, pairs_for, 2 * self.chunk)
        self.exchanges += 1
        lq, gq = self.at[a], self.at[nl + j]
        f = self.flip[j]
        self.at[a], self.at[nl + j] = gq, lq
        self.pos[gq], self.pos[lq] = a, nl + j
        self.flip[j] = 0
        if f:
            for r in self.comm.local_ranks:
                self._emit(r, _inst(K["x"], [a]))

    # -- instructions --
    def _apply_gate(self, inst) -> None:
        kind = int(inst["kind"])
        nq = int(inst["nq"])
        qs = [int(v) for v in inst["q"][:nq]]
        p = np.array(inst["p"], dtype=np.float64)
        if kind == K["swap"]:
            a, b = qs
            pa, pb = self.pos[a], self.pos[b]
            self.pos[a], self.pos[b] = pb, pa
            self.at[pa], self.at[pb] = b, a
            return
        glob = [q for q in qs if self._is_global(q)]
        if not glob:
            for r in self.comm.local_ranks:
                self._emit(r, _inst(kind, [self.pos[q] for q in qs], p))
            return
        if kind in _ONE_Q:
            (q,) = qs
            j = self.pos[q] - self.nl
            if kind == K["x"]:
                self.flip[j] ^= 1
                return
            if kind == K["y"]:
                for r in self.comm.local_ranks:
                    for i in _phase_insts(1j if self._gbit(r, q) == 0 else -1j, 0):
                        self._emit(r, i)
                self.flip[j] ^= 1
                return
            if _phase_1q(kind, p, 0) is not None:
                for r in self.comm.local_ranks:
                    for i in _phase_insts(complex(_phase_1q(kind, p, self._gbit(r, q))), 0):
                        self._emit(r, i)
                return
            self._make_local([q], qs)
            self._emit_local_all(kind, qs, p)
            return
        if kind in _SYM_DIAG and self._is_global(qs[1]) and not self._is_global(qs[0]):
            qs = [qs[1], qs[0]]
        if kind in _SYM_DIAG and self._is_global(qs[0]) and self._is_global(qs[1]):
            ph = -1.0 + 0j if kind in (K["cz"], K["g_cz"]) else complex(math.cos(p[0]), math.sin(p[0]))
            for r in self.comm.local_ranks:
                if self._gbit(r, qs[0]) and self._gbit(r, qs[1]):
                    for i in _phase_insts(ph, 0):
                        self._emit(r, i)
            return
        if kind == K["crz"] and self._is_global(qs[1]):
            c, t = qs
            for r in self.comm.local_ranks:
                e = self._gbit(r, t)
                h = 0.5 * p[0] if e else -0.5 * p[0]
                if self._is_global(c):
                    if self._gbit(r, c):
                        for i in _phase_insts(complex(math.cos(h), math.sin(h)), 0):
                            self._emit(r, i)
                else:
                    self._emit(r, _inst(K["u1"], [self.pos[c]], [h]))
            return
        if kind == K["rzz"]:
            a, b = qs
            for r in self.comm.local_ranks:
                if self._is_global(a) and self._is_global(b):
                    s = 1.0 if self._gbit(r, a) != self._gbit(r, b) else -1.0
                    h = 0.5 * p[0] * s
                    for i in _phase_insts(complex(math.cos(h), math.sin(h)), 0):
                        self._emit(r, i)
                else:
                    gq, lq = (a, b) if self._is_global(a) else (b, a)
                    th = -p[0] if self._gbit(r, gq) else p[0]
                    self._emit(r, _inst(K["rz"], [self.pos[lq]], [th]))
            return
        nctl = _NCTL.get(kind, 0)
        ctl_glob = [q for q in qs[:nctl] if self._is_global(q)]
        if ctl_glob and all(not self._is_global(q) for q in qs[nctl:]):
            for r in self.comm.local_ranks:
                if any(self._gbit(r, q) == 0 for q in ctl_glob):
                    continue
                k2, rest = kind, list(qs)
                for q in ctl_glob:
                    rest.remove(q)
                    k2 = _DROP[k2]
                phase = None
                if kind == K["cu"]:
                    phase = complex(math.cos(p[3]), math.sin(p[3]))
                pp = p[:3] if kind == K["cu"] else p
                self._emit(r, _inst(k2, [self.pos[q] for q in rest], pp))
                if phase is not None:
                    for i in _phase_insts(phase, self.pos[rest[-1]]):
                        self._emit(r, i)
            return
        # a global qubit in a role no reduction covers: make every qubit local
        self._make_local(glob, qs)
        self._emit_local_all(kind, qs, p)

    def _emit_local_all(self, kind: int, qs: Sequence[int], p: np.ndarray) -> None:
        for r in self.comm.local_ranks:
            self._emit(r, _inst(kind, [self.pos[q] for q in qs], p))

    def _measure(self, q: int, draw: float) -> int:
        self._make_local([q], [q])
        self._flush()
        a = self.pos[q]
        parts = [np.array([self.shards[r].p1(a)]) for r in self.comm.local_ranks]
        p1 = float(self.comm.allreduce([np.sum(parts, axis=0)])[0])
        o = 1 if draw < p1 else 0
        if abs(draw - p1) < 1e-12:
            self.boundary_draws += 1
        for r in self.comm.local_ranks:
            self.shards[r].collapse(a, o, p1)
        return o

    def run(self, prog: Program, seed: int) -> np.ndarray:
        """Runs ``prog`` (``simulate`` semantics) from the current state;
        returns the classical bits (-1 = never written)."""
        from .statevector import _unsupported_message

        if prog.num_qubits > self.n:
            raise ValueError("the program has more qubits than the sharded state")
        cbits = np.full(prog.cbit_space, -1, dtype=np.int32)
        draws = 0
        seed &= _U64
        for idx in range(prog.ninst):
            inst = prog.insts[idx]
            if not self._cond_holds(prog, inst, cbits):
                continue
            kind = int(inst["kind"])
            if kind in _NOOP:
                continue
            if kind in (K["g_opaque"], K["g_unsupported"]):
                self._flush()
                raise NotImplementedError(_unsupported_message(prog, idx))
            if kind in (K["measure"], K["reset"]):
                r = float(_rng_f64(seed, draws, 1)[0])
                draws += 1
                q = int(inst["q"][0])
                o = self._measure(q, r)
                if kind == K["measure"]:
                    cbits[int(inst["cbit"])] = o
                elif o == 1:
                    for rr in self.comm.local_ranks:
                        self._emit(rr, _inst(K["x"], [self.pos[q]]))
                continue
            self._apply_gate(inst)
        self._flush()
        return cbits

    @staticmethod
    def _cond_holds(prog: Program, inst, cbits: np.ndarray) -> bool:
        for c in range(int(inst["cond_count"])):
            cd = prog.conds[int(inst["cond_first"]) + c]
            actual = 0
            for b in range(int(cd["creg_size"])):
                i = int(cd["creg_base"]) + b
                if i < cbits.size and cbits[i] > 0:
                    actual |= 1 << b
            if actual != int(cd["creg_value"]):
                return False
        return True

    # -- results --
    def probabilities(self, qubits: Sequence[int]) -> np.ndarray:
        """Marginal probabilities over logical ``qubits`` (qubits[0] = MSB of
        the outcome index), identical on every rank."""
        qs = [int(q) for q in qubits]
        k = len(qs)
        self._flush()
        loc = [q for q in qs if not self._is_global(q)]
        parts = []
        for r in self.comm.local_ranks:
            m = self.shards[r].marginal([self.pos[q] for q in loc]) if loc else np.array(
                [_norm_from_marginal(self.shards[r])])
            full = np.zeros(1 << k, dtype=np.float64)
            # outcome index: bit (k-1-i) is qubit qs[i]
            gidx = 0
            for i, q in enumerate(qs):
                if self._is_global(q) and self._gbit(r, q):
                    gidx |= 1 << (k - 1 - i)
            t = np.arange(m.size, dtype=np.int64)
            idx = np.full(m.size, gidx, dtype=np.int64)
            for bi, q in enumerate(loc):
                idx |= ((t >> (len(loc) - 1 - bi)) & 1) << (k - 1 - qs.index(q))
            full[idx] = m
            parts.append(full)
        return self.comm.allreduce([np.sum(parts, axis=0)])

    def statevector(self) -> np.ndarray:
        """The full logical state gathered on every rank (small n only)."""
        import torch

        self._flush()
        shards = {r: s.download() for r, s in self.shards.items()}
        if isinstance(self.comm, LocalShards):
            allv = [shards[r] for r in range(self.comm.world)]
        else:
            t = torch.from_numpy(shards[self.comm.rank].view(np.float64).copy())
            dev = self.comm._device()
            t = t.to(dev)
            outs = [torch.empty_like(t) for _ in range(self.comm.world)]
            self.comm.dist.all_gather(outs, t, group=self.comm.group)
            allv = [o.cpu().numpy().view(np.complex128) for o in outs]
        phys = np.concatenate(allv)
        x = np.arange(1 << self.n, dtype=np.int64)
        logical = np.zeros_like(x)
        for q in range(self.n):
            b = (x >> self.pos[q]) & 1
            if self.pos[q] >= self.nl:
                b ^= self.flip[self.pos[q] - self.nl]
            logical |= b << q
        out = np.empty_like(phys)
        out[logical] = phys
        return out

    def release(self) -> None:
        for s in self.shards.values():
            s.release()
        self.shards = {}


def _norm_from_marginal(shard) -> float:
    m = shard.marginal([0])
    return float(m[0] + m[1])


def _rng_f64(seed: int, skip: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    nat.check(nat.lib().dq_rng_f64(seed & _U64, skip, count, nat.ptr(out)), "dq_rng_f64")
    return out
