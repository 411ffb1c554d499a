"""The ghost fill inside the stage kernels (MBM_GHOST_SCATTER=1: each work item writes
the ghost cells whose source cells it stored) against the separate gather launch:
every layer, ghost cells included, bit for bit, in both arithmetic modes; on decks with
block interfaces, walls, Dirichlet edges and open edges; in a batch; and in the
frozen-dt replay the adjoint recomputes its segments with."""
import os

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import adjoint as adj, blockfile as bf, scenario as sc, solver as sv

pytestmark = pytest.mark.gpu


def _shrunk(name, k):
    d = H.deck(name)
    d.blocks = [bf.Block(b.block_id, b.xmin, b.xmax, b.ymin, b.ymax, max(6, b.nx // k), max(6, b.ny // k), b.bc)
                for b in d.blocks]
    return d


def _with(value, fn):
    """Run fn with contexts created under MBM_GHOST_SCATTER=value."""
    old = os.environ.get("MBM_GHOST_SCATTER")
    os.environ["MBM_GHOST_SCATTER"] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ["MBM_GHOST_SCATTER"]
        else:
            os.environ["MBM_GHOST_SCATTER"] = old


CASES = [
    ("ffs28", "ffs", 1, 0.01),          # Dirichlet inflow, walls, 28 blocks with interfaces
    ("Lshape", "riemann2d", 3, 0.02),   # walls on the concave edges, interfaces
    ("square4Box", "riemann2d", 4, 0.02),
    ("squareSmall", "riemann2d", 1, 0.05),
]


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("name,scen,shrink,tend", CASES)
def test_steps_scatter_equals_gather(mode, name, scen, shrink, tend):
    d = _shrunk(name, shrink)
    scn = sc.Scenario.named(scen)

    def run():
        with sv.Solver(d, scn, mode=mode) as s:
            s.initialise()
            t, n, r = s.steps(0.0, tend)
            return s.ghost_scatter(), (t, n, r), [[s.download(l, b) for b in range(len(d.blocks))] for l in (0, 1, 2)]

    on, res_s, lay_s = _with("1", run)
    off, res_g, lay_g = _with("0", run)
    assert on and not off
    assert res_s == res_g and res_s[1] > 0
    for l in range(3):
        for b in range(len(d.blocks)):
            H.assert_bitwise(lay_s[l][b], lay_g[l][b], f"layer {l} block {b}")


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_batch_scatter_equals_gather(mode):
    cases = sv.batch_workload(seed=11, ncases=8, nmin=8, nmax=40)

    def run():
        with sv.BatchSolver(cases, mode=mode) as bs:
            bs.initialise()
            t, ns, nr = bs.steps(0.0, 1.0, max_steps=30)
            return (list(t), list(ns), list(nr)), [[bs.download(0, k, b) for b in range(len(dk.blocks))]
                                                    for k, (dk, _) in enumerate(cases)]

    res_s, lay_s = _with("1", run)
    res_g, lay_g = _with("0", run)
    assert res_s == res_g
    for k in range(len(cases)):
        for b in range(len(lay_s[k])):
            H.assert_bitwise(lay_s[k][b], lay_g[k][b], f"case {k} block {b}")


def test_replay_and_adjoint_scatter_equals_gather():
    """Frozen-dt steps (the path the adjoint recomputes its segments on) and the
    adjoint itself."""
    d = H.quadrant_deck(24, Kn=0.01, limiter=bf.LIM_HARMONIC)
    base = adj.smooth_base(d, 3)
    th0 = [1.0 + 0.1 * np.cos(np.linspace(0, 2, b.nx)[None, :] + np.linspace(0, 1, b.ny)[:, None])
           for b in d.blocks]
    dts = np.array([2e-4, 3e-4, 2.5e-4, 3e-4, 2e-4])

    def run():
        with adj.Sensitivity(d, base, mode="fast") as S:
            layers = adj.state_from_theta(d, base, th0)
            S.load(layers)
            Jr = S.replay(dts)
            lay = [S.s.download(sv.L_DATA, b) for b in range(len(d.blocks))]
            on = S.s.ghost_scatter()
            S.load(layers)
            J, g, gK, dts_run, _ = S.run(6, every=2)
            return on, Jr, lay, J, g, gK, dts_run

    on, Jr_s, lay_s, J_s, g_s, gK_s, dt_s = _with("1", run)
    off, Jr_g, lay_g, J_g, g_g, gK_g, dt_g = _with("0", run)
    assert on and not off
    assert Jr_s == Jr_g and J_s == J_g
    H.assert_bitwise(dt_s, dt_g, "dt")
    for b in range(len(d.blocks)):
        H.assert_bitwise(lay_s[b], lay_g[b], f"block {b}")
        assert np.max(np.abs(g_s[b] - g_g[b])) <= 1e-12 * np.max(np.abs(g_g[b]))
    assert abs(gK_s - gK_g) <= 1e-12 * abs(gK_g)
