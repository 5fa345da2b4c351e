"""Test-only emulator of the fused sweep kernel (k_sweep in csrc/dq_fused.cu).

It interprets the encoded sweep programs returned by ``dq_debug_plan``
exactly as the kernel does -- tile gather through the run tables, the
XOR-swizzled shared-memory layout, register phases addressed through the
per-phase lane/warp/register tables, and every op type -- vectorised over
tiles and threads with numpy complex128.  It lets the CPU test suite check
the planner and encoder against the oracle without a GPU; the GPU tests
then check the kernel itself.
"""
from __future__ import annotations

import ctypes
import struct

import numpy as np

from dqsim_bosonic_b200 import _native as nat

OP_U1, OP_U1R, OP_U1X, OP_U2, OP_FLUSH_R, OP_FLUSH_T, OP_GPHASE, OP_U1H, OP_SCALE, OP_HPHASE = range(10)
FL_THR, FL_REG, FL_PRE = 1, 2, 4
MAXM = 12
SWZ_G = {3: 3, 4: 5, 5: 6, 6: 7, 7: 3, 8: 5, 9: 6, 10: 7, 11: 1}


def swz(e: int) -> int:
    g = 0
    for k in range(3, MAXM):
        if (e >> k) & 1:
            g ^= SWZ_G[k]
    return e ^ g


def plan(prog, opts=None) -> tuple[list[bytes], int, list[int], int]:
    """Runs dq_debug_plan; returns (sweep program blobs, RB, final perm, n)."""
    L = nat.lib()
    o = opts or nat.RunOpts(0, nat.EXEC_FUSED, 0, 0, 0, 0)
    need = ctypes.c_uint64(0)
    args = (prog.num_qubits, nat.ptr(prog.insts) if prog.ninst else None, prog.ninst, ctypes.byref(o))
    nat.check(L.dq_debug_plan(*args, None, 0, ctypes.byref(need)), "dq_debug_plan")
    buf = (ctypes.c_uint8 * need.value)()
    nat.check(L.dq_debug_plan(*args, buf, need.value, ctypes.byref(need)), "dq_debug_plan")
    raw = bytes(buf)
    magic, ns, rb, _ = struct.unpack_from("<4I", raw, 0)
    assert magic == 0x4C505144
    perm = list(struct.unpack_from("<64I", raw, 16))
    offs = list(struct.unpack_from(f"<{ns}Q", raw, 16 + 256))
    hdr = 16 + 256 + 8 * ns
    blob = raw[hdr:]
    blobs = []
    for off in offs:
        pb = struct.unpack_from("<I", blob, off + 84)[0]
        blobs.append(blob[off:off + pb])
    return blobs, rb, perm, prog.num_qubits


def _c2(b: bytes, off: int, count: int) -> np.ndarray:
    v = np.frombuffer(b, dtype="<f8", count=2 * count, offset=off)
    return v[0::2] + 1j * v[1::2]


def run_sweep(state: np.ndarray, n: int, blob: bytes) -> None:
    """Apply one encoded sweep to state (complex128, modified in place)."""
    m, rb, nphase, nslots = struct.unpack_from("<4I", blob, 0)
    local = list(struct.unpack_from(f"<{MAXM}I", blob, 16))[:m]
    off_phase, off_op, off_slot, off_slotent, off_data, prog_bytes, tile_xload, run_bits = \
        struct.unpack_from("<8I", blob, 64)
    nruns = 1 << (m - run_bits)
    run_len = 1 << run_bits
    off_runoff, off_runswz = struct.unpack_from("<2I", blob, 96)
    runoff = np.array(struct.unpack_from(f"<{nruns}Q", blob, off_runoff), dtype=np.uint64)
    runswz = np.array(struct.unpack_from(f"<{nruns}I", blob, off_runswz), dtype=np.int64)
    T, R = 1 << m, 1 << rb
    TB = m - rb
    THREADS = 1 << TB
    ntiles = 1 << (n - m)
    # tile bases: zero bits inserted at the local positions
    t = np.arange(ntiles, dtype=np.uint64)
    base = t.copy()
    for p in local:
        p = np.uint64(p)
        lowmask = (np.uint64(1) << p) - np.uint64(1)
        base = ((base >> p) << (p + np.uint64(1))) | (base & lowmask)
    lane = np.arange(run_len, dtype=np.uint64)
    swl = np.array([swz(int(x)) for x in range(run_len)], dtype=np.int64)
    # gather: element (run r, offset) -> smem index runswz[r] ^ swz(offset)
    gidx = base[:, None, None] + runoff[None, :, None] + lane[None, None, :]      # tiles x runs x run_len
    sidx = (runswz[:, None] ^ swl[None, :])                                       # runs x run_len
    smem = np.zeros((ntiles, T), dtype=np.complex128)
    # X gates opening the sweep are folded into the load: element e lands at the slot of e ^ flips
    smem[:, sidx.reshape(-1) ^ tile_xload] = state[gidx.reshape(ntiles, -1).astype(np.int64)]
    # per-tile slots
    slots = np.ones((ntiles, max(nslots, 1)), dtype=np.complex128)
    for s in range(nslots):
        count, start = struct.unpack_from("<2I", blob, off_slot + 32 * s)
        w = np.full(ntiles, _c2(blob, off_slot + 32 * s + 16, 1)[0], dtype=np.complex128)
        for e in range(count):
            eo = off_slotent + 32 * (start + e)
            mask = np.uint64(struct.unpack_from("<Q", blob, eo)[0])
            we = _c2(blob, eo + 16, 1)[0]
            hit = (base & mask) == mask
            w = np.where(hit, w * we, w)
        slots[:, s] = w
    tid = np.arange(THREADS)
    off_gstore = struct.unpack_from("<I", blob, 108)[0] if nphase else 0
    direct = None  # the last phase's straight-to-state writes: (global offsets, values)
    for p in range(nphase):
        po = off_phase + 192 * p
        lanesw = np.array(struct.unpack_from("<32I", blob, po), dtype=np.int64)
        warpsw = np.array(struct.unpack_from("<8I", blob, po + 128), dtype=np.int64)
        V = struct.unpack_from("<4I", blob, po + 160)[:rb]
        ob, oe, xload = struct.unpack_from("<3I", blob, po + 176)
        pt = lanesw[tid & 31] ^ warpsw[tid >> 5]                                   # threads
        X = np.array([pt ^ _xor_bits(j, V) for j in range(R)]).T                   # threads x R
        assert X.max() < T and (X ^ xload).max() < T
        a = smem[:, X ^ xload]            # X gates folded into the load address   # tiles x threads x R
        for o in range(ob, oe):
            _exec(blob, off_op + 32 * o, off_data, a, slots, base, tid, rb)
        if off_gstore and p + 1 == nphase:
            # like the kernel: element j of thread (lane, warp) goes to tile base +
            # glane[lane] + gwarp[warp] + the gV of j's bits
            glane = np.array(struct.unpack_from("<32Q", blob, off_gstore), dtype=np.uint64)
            gwarp = np.array(struct.unpack_from("<8Q", blob, off_gstore + 256), dtype=np.uint64)
            gV = struct.unpack_from("<4Q", blob, off_gstore + 320)[:rb]
            gthr = glane[tid & 31] + gwarp[tid >> 5]                               # threads
            goff = np.array([gthr + np.uint64(sum(v for b, v in enumerate(gV) if (j >> b) & 1))
                             for j in range(R)], dtype=np.uint64).T               # threads x R
            # the writes cover each tile element exactly once, at its own address
            assert sorted(goff.reshape(-1).tolist()) == sorted(
                (runoff[:, None] + lane[None, :]).reshape(-1).tolist())
            direct = (base[:, None, None] + goff[None, :, :], a)
            continue
        smem[:, X] = a
    if direct is not None:
        g, a = direct
        assert int(g.max()) < len(state)
        state[g.reshape(-1).astype(np.int64)] = a.reshape(-1)
        return
    state[gidx.reshape(ntiles, -1).astype(np.int64)] = smem[:, sidx.reshape(-1)]


def _xor_bits(j, V):
    x = 0
    for b, v in enumerate(V):
        if (j >> b) & 1:
            x ^= v
    return x


def _exec(blob, oo, off_data, a, slots, base, tid, rb):
    w0, w1, data = struct.unpack_from("<3I", blob, oo)
    typ, b0, b1, creg = w0 & 0xFF, (w0 >> 8) & 0xFF, (w0 >> 16) & 0xFF, w0 >> 24
    ctl_thr, flags, slot = w1 & 0xFF, (w1 >> 8) & 0xFF, w1 >> 16
    cnl = np.uint64(struct.unpack_from("<Q", blob, oo + 16)[0])
    R = 1 << rb
    tmask = ((base & cnl) == cnl)[:, None]                     # tiles x 1
    hmask = ((tid & ctl_thr) == ctl_thr)[None, :]              # 1 x threads
    act = tmask & hmask                                        # tiles x threads
    D = off_data + 16 * data

    def upd(j, v):
        a[:, :, j] = np.where(act, v, a[:, :, j])

    def flush_factors(T):
        W = np.broadcast_to(slots[:, slot][:, None], act.shape).copy()
        if flags & FL_THR:
            lt = _c2(blob, T, 32)
            wt = _c2(blob, T + 16 * 32, 8)
            W = W * (lt[tid & 31] * wt[tid >> 5])[None, :]
            T = T + 16 * 40
        return W, T

    if flags & FL_PRE:
        W, Fo = flush_factors(D + 16 * 4)
        F = _c2(blob, Fo, 1 << (rb - 1)) if flags & FL_REG else None
        for j in range(R):
            if not (j >> b0) & 1:
                continue
            idx = ((j >> (b0 + 1)) << b0) | (j & ((1 << b0) - 1))
            upd(j, a[:, :, j] * (W * (F[idx] if F is not None else 1.0)))
    if typ in (OP_U1, OP_U1R, OP_U1H, OP_U1X):
        if typ == OP_U1H:
            u = np.array([1, 1, 1, -1], dtype=np.complex128)
        elif typ == OP_U1X:
            u = np.array([0, 1, 1, 0], dtype=np.complex128)
        else:
            u = _c2(blob, D, 4)
            if typ == OP_U1R:
                u = u.real.astype(np.complex128)
        for j in range(R):
            if (j >> b0) & 1 or (j & creg) != creg:
                continue
            k = j | (1 << b0)
            x, y = a[:, :, j].copy(), a[:, :, k].copy()
            upd(j, u[0] * x + u[1] * y)
            upd(k, u[2] * x + u[3] * y)
    elif typ == OP_U2:
        u = _c2(blob, D, 16).reshape(4, 4)
        for j in range(R):
            if j & ((1 << b0) | (1 << b1)) or (j & creg) != creg:
                continue
            idx = [j, j | (1 << b1), j | (1 << b0), j | (1 << b0) | (1 << b1)]
            v = [a[:, :, i].copy() for i in idx]
            for r in range(4):
                upd(idx[r], sum(u[r, c] * v[c] for c in range(4)))
    elif typ in (OP_FLUSH_R, OP_FLUSH_T):
        W, Fo = flush_factors(D)
        if typ == OP_FLUSH_T:
            act = act & ((tid >> b0) & 1).astype(bool)[None, :]
        if typ == OP_FLUSH_R:
            F = _c2(blob, Fo, 1 << (rb - 1)) if flags & FL_REG else None
            for j in range(R):
                if not (j >> b0) & 1:
                    continue
                idx = ((j >> (b0 + 1)) << b0) | (j & ((1 << b0) - 1))
                f = W * (F[idx] if F is not None else 1.0)
                upd(j, a[:, :, j] * f)
        else:
            F = _c2(blob, Fo, R) if flags & FL_REG else None
            for j in range(R):
                f = W * (F[j] if F is not None else 1.0)
                upd(j, a[:, :, j] * f)
    elif typ == OP_GPHASE:
        W = slots[:, slot][:, None]
        for j in range(R):
            upd(j, a[:, :, j] * W)
    elif typ == OP_SCALE:
        f = _c2(blob, D, 1)[0].real
        for j in range(R):
            upd(j, a[:, :, j] * f)
    elif typ == OP_HPHASE:
        # marker of a straight-line H phase: its sub-ops follow as ordinary ops
        # (the kernel folds the trailing scale into the last one: same values)
        assert b1 >= 1 and creg == 0
    else:
        raise AssertionError(f"unknown op {typ}")


def emulate(prog, init: np.ndarray, opts=None) -> tuple[np.ndarray, list[int], int]:
    """Apply the planned sweeps of a unitary program; returns (state in
    physical layout, final perm, number of sweeps)."""
    blobs, rb, perm, n = plan(prog, opts)
    st = np.array(init, dtype=np.complex128, copy=True)
    for b in blobs:
        run_sweep(st, n, b)
    return st, perm[:n], len(blobs)


def canonical(state: np.ndarray, perm: list[int]) -> np.ndarray:
    """Undo a relabeling: logical qubit l is stored at physical bit perm[l]."""
    n = len(perm)
    idx = np.arange(1 << n)
    phys = np.zeros_like(idx)
    for l in range(n):
        phys |= ((idx >> l) & 1) << perm[l]
    return state[phys]
