"""A case split over ranks by block, run as several parts on one GPU (the exchange is a
device copy between the parts, the CFL maximum a device reduction; no part waits on
another inside a kernel): the result equals the unsplit solver's bit for bit, steps,
rejections and end time included."""
import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import _abi
from multiblockmomentsfv_b200 import scenario as sc
from multiblockmomentsfv_b200 import sharded
from multiblockmomentsfv_b200 import solver as sv

pytestmark = pytest.mark.gpu


def _unsplit(d, scn, tend, mode, max_steps=0):
    with sv.Solver(d, scn, mode=mode, show_every=0) as s:
        s.initialise()
        t, n, r = s.steps(0.0, tend, max_steps=max_steps)
        return [s.download(sv.L_DATA, b) for b in range(len(d.blocks))], (t, n, r)


def _split(d, scn, owner, nranks, tend, mode, max_steps=0):
    import torch
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [sharded.ShardPart(d, owner, nranks, r, scn, stream=stream.cuda_stream, mode=mode)
                 for r in range(nranks)]
        try:
            ex = sharded.LocalExchange()
            sharded.initialise(parts, scn, ex)
            res = sharded.steps(parts, ex, 0.0, tend, max_steps=max_steps)
            layers = [None] * len(d.blocks)
            for p in parts:
                for g in p.blocks:
                    layers[g] = p.download(sv.L_DATA, g)
            return layers, res
        finally:
            for p in parts:
                p.close()


CASES = [
    ("quadrant 4 x 96^2, 2 ranks", lambda: (H.quadrant_deck(96, Kn=0.01), sc.Scenario.seeded_quadrant(3)),
     lambda d: sharded.owners_by_cells(d, 2), 2, 0.05),
    ("quadrant 4 x 64^2, 4 ranks", lambda: (H.quadrant_deck(64, Kn=0.005, limiter=3), sc.Scenario.seeded_quadrant(4)),
     lambda d: [0, 1, 2, 3], 4, 0.05),
    ("ffs28 (Dirichlet, walls), 3 ranks round robin", lambda: (H.deck("ffs28"), sc.Scenario.named("ffs")),
     lambda d: [b % 3 for b in range(len(d.blocks))], 3, 0.02),
    ("Lshape, 2 ranks", lambda: (H.deck("Lshape"), sc.Scenario.named("riemann2d")),
     lambda d: sharded.owners_by_cells(d, 2), 2, 0.02),
]


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_split_equals_unsplit(case, mode):
    _, make, own, nranks, tend = case
    d, scn = make()
    owner = own(d)
    ref, (t0, n0, r0) = _unsplit(d, scn, tend, mode)
    got, (t1, n1, r1) = _split(d, scn, owner, nranks, tend, mode)
    assert (t1, n1, r1) == (t0, n0, r0)
    assert n0 > 0
    for b in range(len(d.blocks)):
        H.assert_bitwise(got[b], ref[b], f"block {b + 1}")


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("max_steps,batch", [(5, 8), (13, 4), (7, 1)])
def test_split_step_cap_within_a_batch(mode, max_steps, batch):
    """The split loop enqueues `batch` attempts per host wait; a step cap that falls inside
    a batch leaves the attempts after it as no-ops on the device: the same state, step
    count and time as the unsplit solver capped at the same step, and two calls in a row
    continue where the first stopped."""
    import torch
    d, scn = H.quadrant_deck(40, Kn=0.01, limiter=3), sc.Scenario.seeded_quadrant(6)
    owner = [0, 1, 1, 0]
    with sv.Solver(d, scn, mode=mode, show_every=0) as s:
        s.initialise()
        r1 = s.steps(0.0, 0.1, max_steps=max_steps)
        r2 = s.steps(r1[0], 0.1, max_steps=max_steps)
        ref = [s.download(sv.L_DATA, b) for b in range(len(d.blocks))]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [sharded.ShardPart(d, owner, 2, r, scn, stream=stream.cuda_stream, mode=mode) for r in range(2)]
        try:
            ex = sharded.LocalExchange()
            sharded.initialise(parts, scn, ex)
            g1 = sharded.steps(parts, ex, 0.0, 0.1, max_steps=max_steps, batch=batch)
            g2 = sharded.steps(parts, ex, g1[0], 0.1, max_steps=max_steps, batch=batch)
            got = [None] * len(d.blocks)
            for p in parts:
                for g in p.blocks:
                    got[g] = p.download(sv.L_DATA, g)
        finally:
            for p in parts:
                p.close()
    assert (g1, g2) == (r1, r2) and g1[1] == max_steps
    for b in range(len(d.blocks)):
        H.assert_bitwise(got[b], ref[b], f"block {b + 1}")


def test_split_non_finite_stops_every_rank():
    import torch
    d, scn = H.quadrant_deck(48, Kn=0.01), sc.Scenario.seeded_quadrant(2)
    owner = [0, 0, 1, 1]
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        parts = [sharded.ShardPart(d, owner, 2, r, scn, stream=stream.cuda_stream) for r in range(2)]
        try:
            ex = sharded.LocalExchange()
            sharded.initialise(parts, scn, ex)
            U = parts[1].download(sv.L_DATA, 3)
            U[10, 10, 0] = np.nan
            parts[1].upload(sv.L_DATA, 3, U)
            with pytest.raises(_abi.MBMError) as e:
                sharded.steps(parts, ex, 0.0, 0.05)
            assert e.value.status == _abi.MBM_ENONFINITE
            for p in parts:          # every rank stopped with the status
                with pytest.raises(_abi.MBMError):
                    p.end()
        finally:
            for p in parts:
                p.close()


def test_single_context_calls_refuse_a_part():
    d = H.quadrant_deck(16)
    with sharded.ShardPart(d, [0, 0, 1, 1], 2, 0) as p:
        import ctypes
        t = ctypes.c_double(0.0)
        assert p.L.mbm_steps(p.ctx, ctypes.byref(t), 0.1, 1.0, 0.95, None, None) == _abi.MBM_EINVAL
        assert p.L.mbm_set_boundary(p.ctx, sv.L_DATA, 0.0) == _abi.MBM_EINVAL
