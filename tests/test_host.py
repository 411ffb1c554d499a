"""Host logic without a GPU: the C-ABI library loads and exports its symbols, the
resolved ghost map equals the reference's two-sweep SetBoundary, the deck parser
and the output writer."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import _abi, blockfile as bf, output as out, scenario as sc, solver


def test_library_loads_and_exports_every_header_symbol():
    L = _abi.lib()
    header = open(os.path.join(H.HERE, "..", "include", "mbm_b200.h")).read()
    declared = set(re.findall(r"\b(mbm_[a-z_]+)\s*\(", header))
    assert declared == set(_abi.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name
    assert L.mbm_version() == 1
    assert L.mbm_strerror(_abi.MBM_EINVAL) == b"invalid argument"


def test_create_without_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(_abi.MBMError) as e:
        solver.Solver(H.deck("squareSmall"))
    assert e.value.status == _abi.MBM_ENODEV


def test_stage_noalloc_argument_checks():
    """mbm_stage_noalloc refuses, before any CUDA call, an output that overlaps its
    input or Data0 (an in-place stage), a non-finite or non-positive dt, too many
    blocks and blocks beyond its scratch; the pointers are never dereferenced, so
    plain integers stand in for device addresses."""
    L = _abi.lib()
    d = H.quadrant_deck(40, Kn=0.01, limiter=4)
    descs = _abi.block_descs(d.blocks)
    n = len(d.blocks)
    total = 0
    for b in d.blocks:      # the plane layout's element count (include/mbm_b200.h)
        pitch = (b.nx + 6 + 1 + 3) // 4 * 4
        total += 9 * ((pitch * (b.ny + 6) + 31) // 32 * 32)
    base, nbytes = 1 << 40, total * 8
    in_, d0 = base, base + 4 * nbytes

    def call(inp, data0, out, dt=1e-3, heun=1, blocks=descs, nb=n):
        st = L.mbm_stage_noalloc(blocks, nb, inp, data0, out, 0.01, 0.0, 4, dt, heun, None, None)
        return st, L.mbm_last_error(None).decode()

    for out_ in (in_, in_ + 8, in_ + nbytes - 8, in_ - nbytes + 8):
        st, msg = call(in_, d0, out_)
        assert st == _abi.MBM_EINVAL and "overlaps" in msg, (out_ - in_, msg)
    for out_ in (d0, d0 + nbytes // 2, d0 - nbytes + 8):
        st, msg = call(in_, d0, out_)
        assert st == _abi.MBM_EINVAL and "overlaps" in msg, (out_ - d0, msg)
    st, msg = call(in_, None, in_ + 8, heun=0)
    assert st == _abi.MBM_EINVAL and "overlaps" in msg
    for dt in (float("inf"), float("nan"), 0.0, -1e-3):
        st, msg = call(in_, d0, base + 2 * nbytes, dt=dt)
        assert st == _abi.MBM_EINVAL and "dt" in msg, dt
    many = _abi.block_descs([d.blocks[0]] * 65)
    st, msg = call(in_, d0, base + 2 * nbytes, blocks=many, nb=65)
    assert st == _abi.MBM_EINVAL and "more than 64 blocks" in msg
    big = _abi.block_descs([bf.Block(1, 0.0, 1.0, 0.0, 1.0, 8192, 8192, (0, 0, 0, 0))])
    st, msg = call(in_, d0, base + 2 * nbytes, blocks=big, nb=1)
    assert st == _abi.MBM_EINVAL and "scratch limit (20064 warp work items" in msg
    # disjoint buffers pass every argument check: on a machine without a GPU the call
    # then stops at the device lookup
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        st, msg = call(in_, d0, base + 2 * nbytes)
        assert st == _abi.MBM_ENODEV, msg


@pytest.mark.parametrize("name", ["squareSmall", "square4", "square4Box", "Lshape", "ffs", "ffs28",
                                  "square16Uniform"])
def test_ghost_map_equals_two_sweep_fill(oracle_mod, name):
    """The gather map reproduces SetBoundary bit for bit on the reference decks
    (open, wall, Dirichlet and sync edges, convex and re-entrant corners)."""
    d = H.deck(name)
    if name in ("square4", "Lshape", "square16Uniform", "square4Box"):
        d.blocks = [bf.Block(b.block_id, b.xmin, b.xmax, b.ymin, b.ymax, max(3, b.nx // 10),
                             max(3, b.ny // 10), b.bc) for b in d.blocks]
    _check_map(oracle_mod, d, np.random.default_rng(1))


@pytest.mark.parametrize("seed", range(40))
def test_ghost_map_random_layouts(oracle_mod, seed):
    rng = np.random.default_rng(100 + seed)
    _check_map(oracle_mod, H.random_deck(rng, max_n=7), rng)


def _check_map(oracle_mod, d, rng):
    scn = sc.Scenario.named("ffs")
    orc = oracle_mod.Oracle(d, scn)
    layers = []
    for b, blk in enumerate(d.blocks):
        U = rng.standard_normal((blk.nyp, blk.nxp, bf.NV))
        orc.set_layer(1, b, U)
        layers.append(U.copy())
    orc.set_boundary(1, 0.0)
    entries = solver.ghost_map(d.blocks)
    rows = []
    for b, blk in enumerate(d.blocks):
        for side in range(4):
            if blk.bc[side] <= -2:
                rows.append(sc.dirichlet_edge(scn, blk, side).reshape(-1, bf.NV))
    dirichlet = np.concatenate(rows) if rows else None
    H.apply_ghost_map(entries, layers, dirichlet)
    for b in range(len(d.blocks)):
        H.assert_bitwise(layers[b], orc.get_layer(1, b), f"block {b + 1}")


def test_ghost_map_rejects_bad_tables():
    B = bf.Block
    with pytest.raises(_abi.MBMError):      # partner does not exist
        solver.ghost_map([B(1, 0, 1, 0, 1, 5, 5, (0, 2, 0, 0))])
    with pytest.raises(_abi.MBMError):      # non-conforming interface
        solver.ghost_map([B(1, 0, 1, 0, 1, 5, 5, (0, 2, 0, 0)), B(2, 1, 2, 0, 1, 5, 6, (1, 0, 0, 0))])
    with pytest.raises(_abi.MBMError):      # too narrow: a ghost cell keeps no defined source
        solver.ghost_map([B(1, 0, 1, 0, 1, 1, 5, (-1, -1, 0, 0))])
    with pytest.raises(_abi.MBMError):      # cell size outside (1e-100, 1e100)
        solver.ghost_map([B(1, 0, 1e-200, 0, 1, 5, 5, (-1, -1, 0, 0))])


def test_dirichlet_edge_order():
    blk = bf.Block(1, -1.0, 0.0, -1.0, 1.0, 4, 5, (-2, 0, 0, 0))
    v = sc.dirichlet_edge(sc.Scenario.named("riemann2d"), blk, 0)
    assert v.shape == (blk.nyp, 3, bf.NV)
    x, y = blk.centres()
    ref = sc.initial_state(sc.Scenario.named("riemann2d"), x[4, 3 - 2], y[4, 3 - 2])
    assert np.array_equal(v[4, 1], ref)


def test_deck_parser_reads_every_reference_deck():
    for f in sorted(os.listdir(H.DECKS)):
        d = bf.parse_file(os.path.join(H.DECKS, f))
        assert d.blocks and d.t_out
    d = H.deck("squareSmall")
    assert (d.Kn, d.CFL, d.limiter, d.full_grid_size) == (0.001, 0.95, bf.LIM_HARMONIC, 400)
    assert d.t_out == [0.05, 0.1, 0.15000000000000002, 0.2, 0.25, 0.30000000000000004]
    assert d.blocks[0].x0 == -1.25
    d2 = d.with_cli(Kn="0.01")
    assert d2.Kn == float(np.float32(0.01)) != 0.01
    rt = bf.parse_text(bf.format_deck(H.deck("ffs28")))
    assert rt.blocks == H.deck("ffs28").blocks


def test_convert_names():
    assert out.convert(0.05) == "0p05"
    assert out.convert(0.001) == "0p001"
    assert out.convert(0.3) == "0p3"
    assert out.convert(1.0) == "1p0"


def test_scenario_matches_oracle_state(oracle_mod):
    s = sc.Scenario.seeded_quadrant(3)
    xs = np.linspace(-1, 1, 7)
    for x in xs:
        for y in xs:
            U = np.zeros(9)
            oracle_mod.lib().orc_initial_state(C.byref(oracle_mod.c_scenario(s)), x, y, 0.0,
                                               U.ctypes.data_as(C.POINTER(C.c_double)))
            assert np.array_equal(U, sc.initial_state(s, x, y))


def test_cli_help_and_missing_block_file(capsys):
    """The command line answers -h with its flags and a missing block file with one
    line on stderr and status 1 (no GPU needed for either)."""
    from multiblockmomentsfv_b200 import __main__ as cli
    assert cli.main(["prog", "-h"]) == 0
    assert "-bfile" in capsys.readouterr().out
    assert cli.main(["prog", "-bfile", "no/such/deck.txt"]) == 1
    assert "block file not found" in capsys.readouterr().err


@pytest.mark.parametrize("single", [False, True])
def test_regression_gate_equals_reference_tool(tmp_path, single):
    """output.compare, the package's restatement of the reference's regression gate,
    against the reference's own tools/compare_solution.py (staged by the reference
    build) on result files differing by planted amounts around the gate's threshold,
    at the default tolerances and at zero tolerance."""
    rng = np.random.default_rng(11 + single)
    d = H.quadrant_deck(12, Kn=0.01, limiter=4)
    layers = [H.random_layer(rng, b) for b in d.blocks]
    base = out.Writer(str(tmp_path / "base"), d, "Riemann2D", single=single)
    base.write(layers, 0.0, 0)
    base.write(layers, 0.1, 1)
    abstol, reltol = (1e-6, 1e-5) if single else (1e-10, 1e-8)
    cases = [0.0, 0.5, 0.9, 1.1, 3.0]       # planted difference / threshold at one value
    seen = set()
    for k, f in enumerate(cases):
        w = out.Writer(str(tmp_path / f"c{k}"), d, "Riemann2D", single=single)
        w.write(layers, 0.0, 0)
        w.write(layers, 0.1, 1)
        # plant the difference in one value of the second level's first zone
        _, dat = out.companion(w.base)
        esize = 4 if single else 8
        z = out.read(w.base)[0][len(d.blocks)]
        idx = 37
        y = float(z["values"].ravel()[idx])
        x = np.array([y + f * (abstol + reltol * abs(y))], dtype="<f4" if single else "<f8")
        raw = bytearray(open(dat, "rb").read())
        raw[z["offset"] + idx * esize: z["offset"] + (idx + 1) * esize] = x.tobytes()
        open(dat, "wb").write(bytes(raw))
        ok_pkg, _, msg = out.compare(w.base, base.base)
        ok_ref, log = H.reference_compare(w.base, base.base)
        assert ok_pkg == ok_ref, (f, msg, log)
        seen.add(ok_ref)
        ok0_pkg = out.compare(w.base, base.base, 0.0, 0.0)[0]
        ok0_ref = H.reference_compare(w.base, base.base, 0.0, 0.0)[0]
        assert ok0_pkg == ok0_ref == (f == 0.0), f
    assert seen == {True, False}
