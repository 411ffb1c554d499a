"""One case split over ranks by block (one process per GPU, or several parts in one
process for testing).

Every rank holds the whole block table and an owner per block; `ShardPart` is the
device context of one rank's blocks (mbm_create_sharded).  A Heun attempt runs in
lockstep on all ranks: stage 1, the exchange of the cells other ranks' ghost cells
copy, the ghost fill of TMP, stage 2, exchange, fill of NEW, this rank's CFL, the
maximum over ranks, the controller.  The exchange moves each send buffer's segment
for peer q into q's receive buffer; `DistExchange` does it with torch.distributed
point-to-point messages (NCCL for device buffers), `LocalExchange` with device copies
between parts that live in the same process.  Results equal the unsplit solver's bit
for bit: the ghost map is the same, and a maximum does not depend on its order.

The reference runs every block in one process (src/Main.c:189-244); this is the
split the block structure allows, with one exchange per stage.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _abi
from . import blockfile as bf
from . import scenario as sc
from .solver import L_DATA, L_NEW, L_TMP


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def plan(deck: bf.Deck, owner: Sequence[int], nranks: int, rank: int) -> dict:
    """The exchange plan of one rank (host only): counts per peer and the cells sent
    (global block, cell J*nxp+I) and received (global block, cell, wall flips)."""
    L = _abi.lib()
    descs = _abi.block_descs(deck.blocks)
    own = np.ascontiguousarray(owner, dtype=np.int32)
    sc_ = np.zeros(nranks, dtype=np.int32)
    rc_ = np.zeros(nranks, dtype=np.int32)
    _abi.check(L.mbm_shard_plan(descs, len(deck.blocks), _iptr(own), nranks, rank, _iptr(sc_), _iptr(rc_),
                                None, None, 0))
    cap = int(max(sc_.sum(), rc_.sum(), 1))
    send = np.zeros((cap, 2), dtype=np.int32)
    recv = np.zeros((cap, 3), dtype=np.int32)
    _abi.check(L.mbm_shard_plan(descs, len(deck.blocks), _iptr(own), nranks, rank, _iptr(sc_), _iptr(rc_),
                                _iptr(send), _iptr(recv), cap))
    return {"send_counts": sc_, "recv_counts": rc_, "send": send[:sc_.sum()], "recv": recv[:rc_.sum()]}


def owners_by_cells(deck: bf.Deck, nranks: int) -> List[int]:
    """Blocks to ranks in block order, balancing cell counts (contiguous runs)."""
    cells = np.array([b.cells for b in deck.blocks], dtype=np.float64)
    cum = np.cumsum(cells) - cells / 2
    return [min(nranks - 1, int(c * nranks / cells.sum())) for c in cum]


class _Dev:
    """__cuda_array_interface__ over a device pointer (no copy, no ownership)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


class ShardPart:
    """The device context of one rank's blocks."""

    def __init__(self, deck: bf.Deck, owner: Sequence[int], nranks: int, rank: int,
                 scenario: Optional[sc.Scenario] = None, device: int = 0, stream: Optional[int] = None,
                 mode: str = "exact", show_every: int = 0, segment_rows: int = 0):
        self.deck, self.owner, self.nranks, self.rank = deck, list(owner), nranks, rank
        self.L = _abi.lib()
        self.blocks = [b for b in range(len(deck.blocks)) if self.owner[b] == rank]
        self._local = {g: i for i, g in enumerate(self.blocks)}
        self._descs = _abi.block_descs(deck.blocks)
        p = _abi.Params()
        p.Kn, p.F, p.limiter, p.mode = deck.Kn, deck.F, deck.limiter, _abi.MODES[mode]
        p.device, p.show_every, p.segment_rows = device, show_every, segment_rows
        p.stream = stream
        own = np.ascontiguousarray(self.owner, dtype=np.int32)
        ctx = C.c_void_p()
        st = self.L.mbm_create_sharded(self._descs, len(deck.blocks), _iptr(own), nranks, rank, C.byref(p),
                                       C.byref(ctx))
        if st != _abi.MBM_OK:
            raise _abi.MBMError(st, self.L.mbm_last_error(None).decode())
        self.ctx = ctx
        self.send_counts = np.zeros(nranks, dtype=np.int32)
        self.recv_counts = np.zeros(nranks, dtype=np.int32)
        sp, rp, cp = C.c_void_p(), C.c_void_p(), C.c_void_p()
        self._check(self.L.mbm_shard_buffers(ctx, _iptr(self.send_counts), _iptr(self.recv_counts), nranks,
                                             C.byref(sp), C.byref(rp), C.byref(cp)))
        self._ptrs = (sp.value, rp.value, cp.value)
        self.send_off = np.concatenate([[0], np.cumsum(self.send_counts)]) * bf.NV
        self.recv_off = np.concatenate([[0], np.cumsum(self.recv_counts)]) * bf.NV
        self._views = None
        if scenario is not None:   # every block's Dirichlet edges: corner ghosts may read another rank's
            for g, blk in enumerate(deck.blocks):
                for side in range(4):
                    if blk.bc[side] <= -2:
                        v = np.ascontiguousarray(sc.dirichlet_edge(scenario, blk, side, 0.0))
                        self._check(self.L.mbm_shard_set_dirichlet(self.ctx, g, side, _dptr(v)))

    def _check(self, st: int) -> None:
        _abi.check(st, self.ctx)

    def close(self) -> None:
        if getattr(self, "ctx", None):
            self.L.mbm_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- device buffers as torch tensors (send, recv, cfl) ---------------------
    def views(self):
        if self._views is None:
            import torch
            sp, rp, cp = self._ptrs
            self._views = (torch.as_tensor(_Dev(sp, int(self.send_off[-1]) or 1), device="cuda"),
                           torch.as_tensor(_Dev(rp, int(self.recv_off[-1]) or 1), device="cuda"),
                           torch.as_tensor(_Dev(cp, 1), device="cuda"))
        return self._views

    # -- data, by global block number -----------------------------------------
    def upload(self, layer: int, g: int, U: np.ndarray) -> None:
        U = np.ascontiguousarray(U, dtype=np.float64)
        self._check(self.L.mbm_upload(self.ctx, layer, self._local[g], _dptr(U)))

    def download(self, layer: int, g: int) -> np.ndarray:
        b = self.deck.blocks[g]
        U = np.empty((b.nyp, b.nxp, bf.NV))
        self._check(self.L.mbm_download(self.ctx, layer, self._local[g], _dptr(U)))
        return U

    # -- one phase each ----------------------------------------------------------
    def begin(self, t, tend, CFLmax, CFLreg, max_steps):
        self._check(self.L.mbm_shard_begin(self.ctx, t, tend, CFLmax, CFLreg, max_steps))

    def stage(self, heun: int):
        self._check(self.L.mbm_shard_stage(self.ctx, heun))

    def pack(self, layer: int):
        self._check(self.L.mbm_shard_pack(self.ctx, layer))

    def fill(self, layer: int):
        self._check(self.L.mbm_shard_fill(self.ctx, layer))

    def cfl(self):
        self._check(self.L.mbm_shard_cfl(self.ctx))

    def control(self, wait: bool = True) -> Optional[int]:
        """The controller of the attempt; wait=False enqueues it and returns None."""
        if not wait:
            self._check(self.L.mbm_shard_control(self.ctx, None))
            return None
        d = C.c_int(0)
        self._check(self.L.mbm_shard_control(self.ctx, C.byref(d)))
        return d.value

    def end(self):
        t = C.c_double(0.0)
        n, r = C.c_int(0), C.c_int(0)
        self._check(self.L.mbm_shard_end(self.ctx, C.byref(t), C.byref(n), C.byref(r)))
        return t.value, n.value, r.value


class LocalExchange:
    """All ranks' parts in this process (one device): device-to-device copies on the
    current stream, which the parts must share."""

    def move(self, parts: Sequence[ShardPart]) -> None:
        for p in parts:
            send = p.views()[0]
            for q in parts:
                if q is p or p.send_counts[q.rank] == 0:
                    continue
                recv = q.views()[1]
                a, b = int(p.send_off[q.rank]), int(p.send_off[q.rank + 1])
                c0 = int(q.recv_off[p.rank])
                recv[c0:c0 + (b - a)].copy_(send[a:b])

    def reduce_max(self, parts: Sequence[ShardPart]) -> None:
        import torch
        m = torch.stack([p.views()[2][0] for p in parts]).max()
        for p in parts:
            p.views()[2][0] = m


def exchange_segments(send, recv, send_off, recv_off, rank: int, nranks: int, group=None) -> None:
    """Point-to-point exchange of per-peer segments (torch.distributed; NCCL for CUDA
    tensors, gloo for CPU tensors): segment q of `send` to rank q, segment p of `recv`
    from rank p."""
    import torch.distributed as dist
    ops = []
    for q in range(nranks):
        if q == rank:
            continue
        a, b = int(send_off[q]), int(send_off[q + 1])
        if b > a:
            ops.append(dist.P2POp(dist.isend, send[a:b], q, group))
        c, d = int(recv_off[q]), int(recv_off[q + 1])
        if d > c:
            ops.append(dist.P2POp(dist.irecv, recv[c:d], q, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


class DistExchange:
    """One part per process; the peers are the other ranks of the process group."""

    def __init__(self, group=None):
        self.group = group

    def move(self, parts: Sequence[ShardPart]) -> None:
        (p,) = parts
        send, recv, _ = p.views()
        exchange_segments(send, recv, p.send_off, p.recv_off, p.rank, p.nranks, self.group)

    def reduce_max(self, parts: Sequence[ShardPart]) -> None:
        import torch.distributed as dist
        (p,) = parts
        dist.all_reduce(p.views()[2], op=dist.ReduceOp.MAX, group=self.group)


def boundary(parts: Sequence[ShardPart], ex, layer: int = L_DATA) -> None:
    """SetBoundary of a layer across the ranks (pack, exchange, fill)."""
    for p in parts:
        p.pack(layer)
    ex.move(parts)
    for p in parts:
        p.fill(layer)


def initialise(parts: Sequence[ShardPart], scenario: sc.Scenario, ex) -> None:
    """Initial state of every owned block, then the ghost fill across ranks."""
    for p in parts:
        for g in p.blocks:
            p.upload(L_DATA, g, sc.initial_block(scenario, p.deck.blocks[g]))
    boundary(parts, ex, L_DATA)


def steps(parts: Sequence[ShardPart], ex, t: float, tend: float, CFLmax: float = 1.0,
          CFLreg: Optional[float] = None, max_steps: int = 0, batch: int = 8):
    """Steps() over the split case; returns (t, accepted steps, rejected attempts).
    Attempts are enqueued `batch` at a time, and the host reads the end flag once per
    batch (attempts after the last one return at once on the device); every rank
    enqueues the same attempts, exchanges and reductions."""
    CFLreg = parts[0].deck.CFL if CFLreg is None else CFLreg
    for p in parts:
        p.begin(t, tend, CFLmax, CFLreg, max_steps)
    done = not (t < tend)
    nb = max(1, batch)
    while not done:
        for k in range(nb):
            for heun, out in ((0, L_TMP), (1, L_NEW)):
                for p in parts:
                    p.stage(heun)
                for p in parts:
                    p.pack(out)
                ex.move(parts)
                for p in parts:
                    p.fill(out)
            for p in parts:
                p.cfl()
            ex.reduce_max(parts)
            flags = [p.control(wait=k == nb - 1) for p in parts]
        if len(set(flags)) != 1:
            raise RuntimeError("ranks disagree on the end of the step loop")
        done = bool(flags[0])
    res = [p.end() for p in parts]
    return res[0]
