"""Parity of the CUDA path with the oracle, through the C ABI.

Bitwise mode: every comparison is exact (bit patterns of doubles, signed zeros
included): the stage update, the ghost fill, TimeUpdate with its CFL, whole
Steps intervals with their step counts and progress traces, and the reference
goldens.
"""
import json
import os

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import blockfile as bf, output as out, scenario as sc, solver as sv
from multiblockmomentsfv_b200 import _abi

pytestmark = pytest.mark.gpu


def _pair(oracle_mod, d, scn, rng, layers=(0, 1, 2)):
    orc = oracle_mod.Oracle(d, scn)
    gpu = sv.Solver(d, scn)
    for b, blk in enumerate(d.blocks):
        for l in layers:
            U = H.random_layer(rng, blk)
            orc.set_layer(l, b, U)
            gpu.upload(l, b, U)
    return orc, gpu


@pytest.mark.parametrize("seed", range(10))
def test_stage_update_bitwise(oracle_mod, seed):
    rng = np.random.default_rng(seed)
    d = H.random_deck(rng, max_n=40)
    d.limiter = seed % 5
    d.F = 0.25 if seed % 3 == 0 else 0.0
    orc, gpu = _pair(oracle_mod, d, sc.Scenario.named("riemann2d"), rng)
    dt = 0.004
    with gpu:
        for heun, (o_l, i_l, d0_l) in ((0, (1, 0, 0)), (1, (2, 1, 0))):
            if heun == 1:
                # the oracle's stage 1 also wrote TMP's ghost cells (the fill between
                # stages overwrites them); give both sides the same stage-2 input
                for b in range(len(d.blocks)):
                    gpu.upload(1, b, orc.get_layer(1, b))
            cfl = gpu.update(o_l, i_l, d0_l, dt, 0.2, heun)
            for b in range(len(d.blocks)):
                c = orc.update(b, o_l, i_l, d0_l, dt, 0.2, heun)
                assert np.float64(c).view(np.uint64) == np.float64(cfl[b]).view(np.uint64), (heun, b, c, cfl[b])
                H.assert_bitwise(H.interior(gpu.download(o_l, b)), H.interior(orc.get_layer(o_l, b)),
                                 f"stage {heun} block {b}")


@pytest.mark.parametrize("name", ["square4Box", "Lshape", "ffs28"])
def test_set_boundary_bitwise(oracle_mod, name):
    rng = np.random.default_rng(5)
    d = H.deck(name)
    d.blocks = [bf.Block(b.block_id, b.xmin, b.xmax, b.ymin, b.ymax, max(3, b.nx // 7), max(3, b.ny // 7), b.bc)
                for b in d.blocks]
    orc, gpu = _pair(oracle_mod, d, sc.Scenario.named("ffs"), rng)
    with gpu:
        for l in (0, 1, 2):
            orc.set_boundary(l, 0.0)
            gpu.set_boundary(l, 0.0)
            for b in range(len(d.blocks)):
                H.assert_bitwise(gpu.download(l, b), orc.get_layer(l, b), f"layer {l} block {b}")


@pytest.mark.parametrize("name,limiter", [("squareSmall", 4), ("square4Box", 3), ("Lshape", 2), ("ffs", 1)])
def test_time_update_bitwise(oracle_mod, name, limiter):
    rng = np.random.default_rng(7)
    d = H.deck(name, limiter=limiter)
    d.blocks = [bf.Block(b.block_id, b.xmin, b.xmax, b.ymin, b.ymax, max(3, b.nx // 5), max(3, b.ny // 5), b.bc)
                for b in d.blocks]
    orc, gpu = _pair(oracle_mod, d, sc.Scenario.named("riemann2d"), rng, layers=(0,))
    with gpu:
        orc.set_boundary(0, 0.0)
        gpu.set_boundary(0, 0.0)
        for k in range(4):
            c_o = orc.time_update(0.001, 0.001 * k)
            c_g = gpu.time_update(0.001, 0.001 * k)
            assert c_o == c_g
            for b in range(len(d.blocks)):
                U = orc.get_layer(2, b)
                H.assert_bitwise(gpu.download(2, b), U, f"step {k} block {b}")
                orc.set_layer(0, b, U)
                gpu.upload(0, b, U)


def test_squareSmall_golden_bitwise(tmp_path):
    """reference/squareSmall.ref, all 7 levels, Float32 bit for bit, 112 steps."""
    d = H.deck("squareSmall")
    w, n = sv.run(d, sc.Scenario.named("riemann2d"), str(tmp_path), verbose=False)
    assert n == 112
    zones, _ = out.read(w.hdr)
    g = np.load(os.path.join(H.GOLDEN, "squareSmall_ref.npz"))
    mine = np.concatenate([z["values"].astype(np.float32).ravel() for z in zones])
    assert [z["strand"] for z in zones] == list(g["strand"])
    assert np.array_equal(mine.view(np.uint32), g["values"].view(np.uint32))


def test_square4_golden_bitwise():
    """reference/square4.ref at t = 0.3 bit for bit, 352 steps, and the golden
    console trace (step, CFL, time, next dt every 20 steps)."""
    d = H.deck("square4")
    ref = json.load(open(os.path.join(H.GOLDEN, "square4_ref_trace.json")))
    recs = []
    with sv.Solver(d, sc.Scenario.named("riemann2d")) as s:
        s.initialise()
        t, total = 0.0, 0
        for k, tn in enumerate(d.t_out):
            t, n, rej = s.steps(t, tn)
            total += n
            recs += [(k, int(r[0]), r[1], r[2], r[3]) for r in s.trace()]
        layers = s.layers()
    assert total == 352
    assert len(recs) == len(ref["records"])
    for a, b in zip(recs, ref["records"]):
        assert a[:2] == tuple(b[:2])
        assert ["%f" % v for v in a[2:]] == ["%f" % v for v in b[2:]]
    g = np.load(os.path.join(H.GOLDEN, "square4_ref_t0p3.npz"))
    vals = np.concatenate([out.physical_fields(U[2:-2, 2:-2]).transpose(1, 0, 2).astype(np.float32).ravel()
                           for U in layers])
    assert np.array_equal(vals.view(np.uint32), g["values"].view(np.uint32))


@pytest.mark.parametrize("limiter", range(5))
def test_steps_quadrant_bitwise(oracle_mod, limiter):
    """Seeded quadrant state on the scaled square4 layout (open outer edges), Kn =
    0.01: a whole Steps interval equals the oracle's bit for bit, with the same
    accepted and rejected step counts and progress records."""
    d = H.quadrant_deck(40, Kn=0.01, limiter=limiter)
    scn = sc.Scenario.seeded_quadrant(limiter)
    orc = oracle_mod.Oracle(d, scn)
    orc.initialise()
    t_o, n_o, r_o, tr_o = orc.steps(0.0, 0.05, show_every=5)
    with sv.Solver(d, scn, show_every=5) as s:
        s.initialise()
        t_g, n_g, r_g = s.steps(0.0, 0.05)
        tr_g = s.trace()
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(0, b), orc.get_layer(0, b), f"block {b}")
    assert (t_o, n_o, r_o) == (t_g, n_g, r_g)
    H.assert_bitwise(tr_g, tr_o, "trace")


def test_rejection_path_bitwise(oracle_mod):
    """CFLreg = CFLmax = 1 puts every step at the acceptance threshold, so many
    attempts are rejected: the retry arithmetic matches too.  (CFLreg > CFLmax would
    make the reference retry forever.)"""
    d = H.quadrant_deck(24, Kn=0.003, limiter=3)
    scn = sc.Scenario.seeded_quadrant(9)
    orc = oracle_mod.Oracle(d, scn)
    orc.initialise()
    t_o, n_o, r_o, _ = orc.steps(0.0, 0.02, CFLmax=1.0, CFLreg=1.0)
    assert n_o > 0
    with sv.Solver(d, scn, max_attempts=100000) as s:
        s.initialise()
        t_g, n_g, r_g = s.steps(0.0, 0.02, CFLmax=1.0, CFLreg=1.0)
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(0, b), orc.get_layer(0, b), f"block {b}")
    assert r_o > 0
    assert (t_o, n_o, r_o) == (t_g, n_g, r_g)


def test_dirichlet_and_walls_bitwise(oracle_mod):
    """Forward-facing step with Dirichlet inflow, walls and 28 blocks."""
    d = H.deck("ffs28")
    scn = sc.Scenario.named("ffs")
    orc = oracle_mod.Oracle(d, scn)
    orc.initialise()
    t_o, n_o, r_o, _ = orc.steps(0.0, 0.01)
    with sv.Solver(d, scn) as s:
        s.initialise()
        t_g, n_g, r_g = s.steps(0.0, 0.01)
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(0, b), orc.get_layer(0, b), f"block {b}")
    assert (t_o, n_o, r_o) == (t_g, n_g, r_g)


@pytest.mark.parametrize("limiter", [bf.LIM_AVERAGE, bf.LIM_HARMONIC])
def test_ffs28_refined_bitwise(oracle_mod, limiter):
    """The 28-block forward-facing step refined 4 times (28 blocks of 120 x 40 cells:
    several strips and row segments per block, Dirichlet inflow, walls, 44 interfaces):
    25 steps equal the oracle's bit for bit, both step loops (graph and host-driven)."""
    d = bf.parse_file(os.path.join(H.DECKS, "ffs28.txt"), refine=4)
    d.limiter = limiter
    scn = sc.Scenario.named("ffs")
    orc = oracle_mod.Oracle(d, scn)
    orc.initialise()
    t_o, n_o, r_o, _ = orc.steps(0.0, 1.0, max_steps=25)
    for host_loop in ("0", "1"):
        os.environ["MBM_HOST_LOOP"] = host_loop
        try:
            with sv.Solver(d, scn) as s:
                s.initialise()
                t_g, n_g, r_g = s.steps(0.0, 1.0, max_steps=25)
                for b in range(len(d.blocks)):
                    H.assert_bitwise(s.download(0, b), orc.get_layer(0, b), f"block {b}")
        finally:
            del os.environ["MBM_HOST_LOOP"]
        assert (t_o, n_o, r_o) == (t_g, n_g, r_g)


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_dependent_launch_same_bits(mode):
    """The step loop with programmatic dependent launch (the default) and without it
    (MBM_PDL=0) gives the same layers bit for bit."""
    d = H.quadrant_deck(48, Kn=0.01, limiter=bf.LIM_HARMONIC)
    scn = sc.Scenario.seeded_quadrant(31)
    out = {}
    for pdl in ("1", "0"):
        os.environ["MBM_PDL"] = pdl
        try:
            with sv.Solver(d, scn, mode=mode) as s:
                s.initialise()
                res = s.steps(0.0, 1.0, max_steps=40)
                out[pdl] = (s.dependent_launch(), res, [s.download(l, b) for l in (0, 1, 2)
                                                        for b in range(len(d.blocks))])
        finally:
            del os.environ["MBM_PDL"]
    assert out["1"][0] and not out["0"][0]
    assert out["1"][1] == out["0"][1]
    for a, b in zip(out["1"][2], out["0"][2]):
        H.assert_bitwise(a, b, "layer")


def test_full_size_step_bitwise(oracle_mod):
    """One Heun step (TimeUpdate) of the full benchmark workload (4 blocks x 1024^2,
    seeded quadrant state, Kn = 0.01, harmonic) equals the oracle bit for bit."""
    d = H.quadrant_deck(1024, Kn=0.01)
    scn = sc.Scenario.seeded_quadrant(2024)
    orc = oracle_mod.Oracle(d, scn)
    orc.initialise()
    c_o = orc.time_update(1e-4, 0.0)
    with sv.Solver(d, scn) as s:
        s.initialise()
        c_g = s.time_update(1e-4, 0.0)
        assert c_o == c_g
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(2, b), orc.get_layer(2, b), f"block {b}")
    orc.close()


def test_step_limit_reports_status():
    d = H.quadrant_deck(16)
    with sv.Solver(d, sc.Scenario.seeded_quadrant(1), max_attempts=3) as s:
        s.initialise()
        with pytest.raises(_abi.MBMError) as e:
            s.steps(0.0, 10.0)
        assert e.value.status == _abi.MBM_ESTEPLIMIT


def test_repeatable_bits():
    """Two runs of the same interval give identical bits (no atomics in values)."""
    d = H.quadrant_deck(200, Kn=0.01)
    scn = sc.Scenario.seeded_quadrant(4)
    res = []
    for _ in range(2):
        with sv.Solver(d, scn) as s:
            s.initialise()
            s.steps(0.0, 0.01)
            res.append(s.layers())
    for a, b in zip(*res):
        H.assert_bitwise(a, b, "repeat")
