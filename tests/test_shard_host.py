"""The block split over ranks, on the CPU: the exchange plan (mbm_shard_plan) against
the reference's two-sweep ghost fill (the C oracle), and the point-to-point exchange
of the plan's segments between two gloo ranks."""
import os

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import blockfile as bf
from multiblockmomentsfv_b200 import scenario as sc
from multiblockmomentsfv_b200 import sharded
from multiblockmomentsfv_b200 import solver

NV = bf.NV
SX = np.ones(NV)
SX[[1, 5, 7]] = -1
SY = np.ones(NV)
SY[[2, 5, 8]] = -1


def _flip(v, flags):
    if flags & 1:
        v = v * SX
    if flags & 2:
        v = v * SY
    return v


def _filled(oracle_mod, d, seed):
    """Seeded rough interiors and the oracle's two-sweep fill of them."""
    rng = np.random.default_rng(seed)
    orc = oracle_mod.Oracle(d, sc.Scenario.named("ffs"))
    raw = []
    for b, blk in enumerate(d.blocks):
        U = H.random_layer(rng, blk)
        raw.append(U)
        orc.set_layer(1, b, U)
    orc.set_boundary(1, 0.0)
    full = [orc.get_layer(1, b) for b in range(len(d.blocks))]
    orc.close()
    return raw, full


def _small(name):
    d = H.deck(name)
    if name in ("square4", "Lshape", "square16Uniform", "square4Box"):
        d.blocks = [bf.Block(b.block_id, b.xmin, b.xmax, b.ymin, b.ymax, max(3, b.nx // 10),
                             max(3, b.ny // 10), b.bc) for b in d.blocks]
    return d


def _owner_tables(d):
    nb = len(d.blocks)
    out = []
    for nr in (2, 3, 4):
        if nr > nb:
            continue
        out.append((nr, sharded.owners_by_cells(d, nr)))
        out.append((nr, [b % nr for b in range(nb)]))
    return out


@pytest.mark.parametrize("name", ["square4", "square4Box", "Lshape", "ffs28", "square16Uniform"])
def test_plan_delivers_the_two_sweep_values(oracle_mod, name):
    """For every split: what rank p sends rank r, with the wall flips of r's entries,
    is the value the reference's SetBoundary leaves in r's ghost cells; the counts of
    the two sides agree; every ghost cell with a source on another rank is covered."""
    d = _small(name)
    raw, full = _filled(oracle_mod, d, 5)
    gm = solver.ghost_map(d.blocks)
    for nr, owner in _owner_tables(d):
        plans = [sharded.plan(d, owner, nr, r) for r in range(nr)]
        for r in range(nr):
            pr = plans[r]
            remote = [(db, dc) for db, dc, src, sf in gm
                      if owner[db] == r and src >= 0 and owner[sf & 0xFFFF] != r]
            assert pr["recv"].shape[0] == len(remote)
            roff = np.concatenate([[0], np.cumsum(pr["recv_counts"])])
            for p in range(nr):
                pp = plans[p]
                assert pp["send_counts"][r] == pr["recv_counts"][p]
                soff = np.concatenate([[0], np.cumsum(pp["send_counts"])])
                snd = pp["send"][soff[r]:soff[r + 1]]
                rcv = pr["recv"][roff[p]:roff[p + 1]]
                for (sb, scell), (db, dcell, fl) in zip(snd, rcv):
                    assert owner[sb] == p and owner[db] == r
                    v = _flip(raw[sb].reshape(-1, NV)[scell], fl)
                    assert np.array_equal(v, full[db].reshape(-1, NV)[dcell])
            # a rank sends nothing to itself
            assert pr["send_counts"][r] == 0 and pr["recv_counts"][r] == 0


def test_plan_rejects_bad_owner_tables():
    d = _small("square4")
    with pytest.raises(Exception):
        sharded.plan(d, [0, 1, 2, 5], 4, 0)
    with pytest.raises(Exception):
        sharded.plan(d, [0, 0, 1, 1], 2, 2)


def _gloo_rank(rank, world, port, name, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle as O
        d = _small(name)
        raw, full = _filled(O, d, 9)
        owner = sharded.owners_by_cells(d, world)
        pl = sharded.plan(d, owner, world, rank)
        send = torch.tensor(np.concatenate(
            [raw[b].reshape(-1, NV)[c] for b, c in pl["send"]]) if len(pl["send"]) else np.zeros(1))
        recv = torch.zeros(max(1, int(pl["recv_counts"].sum()) * NV), dtype=torch.float64)
        soff = np.concatenate([[0], np.cumsum(pl["send_counts"])]) * NV
        roff = np.concatenate([[0], np.cumsum(pl["recv_counts"])]) * NV
        sharded.exchange_segments(send, recv, soff, roff, rank, world)
        ok = True
        for k, (db, dc, fl) in enumerate(pl["recv"]):
            v = _flip(recv[k * NV:(k + 1) * NV].numpy(), fl)
            ok = ok and np.array_equal(v, full[db].reshape(-1, NV)[dc])
        q.put((rank, ok, int(pl["recv_counts"].sum())))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("square4", 2), ("ffs28", 2), ("ffs28", 3)])
def test_gloo_exchange_fills_remote_ghosts(name, world):
    """world ranks (processes, gloo): each packs the cells its plan sends, the
    segments travel by isend/irecv, and each rank's received cells equal the
    reference fill of its remote ghost cells."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res), res
    assert sum(n for _, _, n in res) > 0
