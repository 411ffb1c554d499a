"""Output staged on the device (mbm_output_fields) against the host-side payload of
the downloaded state, and failure detection: a NaN in the state ends mbm_steps with
MBM_ENONFINITE instead of running on."""
import os

import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import _abi, output, solver
from multiblockmomentsfv_b200 import scenario as sc
from multiblockmomentsfv_b200 import solver as sv

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("single", [True, False])
def test_output_fields_equal_host_payload(single):
    d = H.random_deck(np.random.default_rng(7))
    with solver.Solver(d, sc.Scenario.named("riemann2d")) as s:
        s.initialise()
        s.steps(0.0, 0.02)
        for b, blk in enumerate(d.blocks):
            host = output.zone_payload(s.download(solver.L_DATA, b), blk.nx, blk.ny, single)
            dev = s.output_fields(b, single).tobytes()
            assert dev == host, f"block {b + 1}"


def test_writer_from_device_writes_identical_files(tmp_path):
    d = H.quadrant_deck(40, Kn=0.01, limiter=2)
    with solver.Solver(d, sc.Scenario.seeded_quadrant(4)) as s:
        s.initialise()
        w_host = output.Writer(str(tmp_path / "host"), d, "Quadrant")
        w_dev = output.Writer(str(tmp_path / "dev"), d, "Quadrant")
        t = 0.0
        for k, tend in enumerate([0.01, 0.02]):
            t, _, _ = s.steps(t, tend)
            w_host.write(s.layers(), t, k)
            w_dev.write_solver(s, t, k)
    with open(w_host.dat, "rb") as a, open(w_dev.dat, "rb") as b:
        assert a.read() == b.read()
    ok, mx, msg = output.compare(w_dev.base, w_host.base, 0.0, 0.0)
    assert ok and mx == 0.0, msg


@pytest.mark.parametrize("mode,bad,comp", [("exact", np.nan, 3), ("fast", np.nan, 3), ("fast", -np.inf, 7),
                                           ("exact", -np.nan, 0)])
def test_nan_in_state_is_reported(mode, bad, comp):
    """A NaN or infinity (either sign) in one moment of one cell ends the step loop
    with MBM_ENONFINITE in both arithmetic modes."""
    d = H.quadrant_deck(32, Kn=0.01)
    with solver.Solver(d, sc.Scenario.seeded_quadrant(2), mode=mode) as s:
        s.initialise()
        U = s.download(solver.L_DATA, 1)
        U[10, 12, comp] = bad
        s.upload(solver.L_DATA, 1, U)
        with pytest.raises(_abi.MBMError) as e:
            s.steps(0.0, 0.05)
        assert e.value.status == _abi.MBM_ENONFINITE
        # the context stays usable: a clean state steps again
        s.initialise()
        t, n, _ = s.steps(0.0, 0.01)
        assert n > 0 and abs(t - 0.01) < 1e-15


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_batch_nonfinite_case_stops_alone(mode):
    """In a batch, a case that goes non-finite stops with MBM_ENONFINITE while the
    others run to the end with the results they have alone."""
    cases = [(H.quadrant_deck(24, Kn=0.01), sc.Scenario.seeded_quadrant(k)) for k in range(3)]
    with solver.BatchSolver(cases, mode=mode) as bs:
        bs.initialise()
        U = bs.download(solver.L_DATA, 1, 2)
        U[8, 9, 0] = np.inf
        bs.upload(solver.L_DATA, 1, 2, U)
        with pytest.raises(_abi.MBMError) as e:
            bs.steps(0.0, 0.02)
        assert e.value.status == _abi.MBM_ENONFINITE
        bs.initialise()
        bs.upload(solver.L_DATA, 1, 2, U)
        t, ns, _ = bs.steps(0.0, 0.02, check=False)
        st = bs.case_status()
        assert list(st) == [_abi.MBM_OK, _abi.MBM_ENONFINITE, _abi.MBM_OK]
        assert ns[1] == 0 and abs(t[0] - 0.02) < 1e-15 and abs(t[2] - 0.02) < 1e-15
        ref = [bs.download(solver.L_DATA, k, b) for k in (0, 2) for b in range(4)]
    for i, k in enumerate((0, 2)):
        with solver.Solver(cases[k][0], cases[k][1], mode=mode) as s:
            s.initialise()
            s.steps(0.0, 0.02)
            for b in range(4):
                H.assert_bitwise(s.download(solver.L_DATA, b), ref[4 * i + b], f"case {k} block {b + 1}")


def _zone_lines(hdr):
    with open(hdr) as f:
        return [line for line in f if line.startswith("ZONE")]


def test_overlapped_output_writes_the_same_files(tmp_path):
    """run() with each interval's output copied beside the next interval and written
    while it runs: the same .dat bytes and ZONE records as the step-then-write loop."""
    d = H.deck("squareSmall")
    scn = sc.Scenario.named("riemann2d")
    wa, na = solver.run(d, scn, str(tmp_path / "a"), single=False, verbose=False, overlap=False)
    wb, nb = solver.run(d, scn, str(tmp_path / "b"), single=False, verbose=False, overlap=True)
    assert na == nb
    with open(wa.dat, "rb") as a, open(wb.dat, "rb") as b:
        assert a.read() == b.read()
    assert _zone_lines(wa.hdr) == _zone_lines(wb.hdr)


def test_cli_matches_the_reference_binary(tmp_path):
    """python -m multiblockmomentsfv_b200 (the Python mirror of main) on the reference's
    own deck writes the files the reference binary writes, bit for bit (-double)."""
    import subprocess
    import sys
    ref = os.path.join(H.HERE, "..", "oracle", "_ref", "moments")
    deck = os.path.join(H.DECKS, "squareSmall.txt")
    r = subprocess.run([sys.executable, "-m", "multiblockmomentsfv_b200", "-bfile", deck, "-out",
                        str(tmp_path / "cli"), "-double"], capture_output=True, text=True, timeout=600,
                       cwd=os.path.join(H.HERE, ".."))
    assert r.returncode == 0, r.stderr[-2000:]
    got = [f for f in os.listdir(tmp_path / "cli") if f.endswith(".hdr")]
    assert len(got) == 1
    if not os.path.exists(ref):
        pytest.skip("reference binary not built (make -C oracle ref)")
    env = dict(os.environ, MBM_SCENARIO="riemann2d", OMP_NUM_THREADS="1")
    r2 = subprocess.run([ref, "-bfile", deck, "-out", str(tmp_path / "ref"), "-double"], env=env,
                        capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0
    ok, mx, msg = output.compare(str(tmp_path / "cli" / got[0]), str(tmp_path / "ref" / got[0]), 0.0, 0.0)
    assert ok and mx == 0.0, msg


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("faithful", [False, True])
def test_device_restart_load_equals_host_loaddata(tmp_path, single, faithful):
    """mbm_load_fields (LoadData on the device) against the host restart loader, which
    equals the reference's own LoadData bit for bit (tests/test_restart.py): every cell of
    L_DATA, both mappings, both payload precisions, on a two-level file."""
    from multiblockmomentsfv_b200 import __main__ as cli
    rng = np.random.default_rng(21 + 2 * single + faithful)
    d = H.deck("Lshape")
    lv = [[H.random_layer(rng, b) for b in d.blocks] for _ in range(2)]
    w = output.Writer(str(tmp_path), d, "Riemann2D", single=single)
    w.write(lv[0], 0.0, -1)
    w.write(lv[1], 0.1, 5)
    want = cli.load_restart(d, w.base, faithful=faithful)
    payloads = cli.restart_payloads(d, w.base, faithful=faithful)
    assert all(p.dtype == (np.float32 if single else np.float64) for p in payloads)
    with sv.Solver(d, sc.Scenario.named("riemann2d")) as s:
        for b in range(len(d.blocks)):
            s.upload(sv.L_DATA, b, np.full((d.blocks[b].nyp, d.blocks[b].nxp, 9), 7.0))   # overwritten
            s.load_fields(b, payloads[b], faithful)
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(sv.L_DATA, b), want[b], f"block {b + 1}")


def test_cli_restart_matches_the_reference_binary(tmp_path):
    """-sfile through the Python mirror of main (the restart loaded on the device) and
    through the reference binary (its own LoadData, CPU steps): identical files."""
    import subprocess
    import sys
    ref = os.path.join(H.HERE, "..", "oracle", "_ref", "moments")
    if not os.path.exists(ref):
        pytest.skip("reference binary not built (make -C oracle ref)")
    env = dict(os.environ, MBM_SCENARIO="riemann2d", OMP_NUM_THREADS="1")
    text = open(os.path.join(H.DECKS, "squareSmall.txt")).read().splitlines()
    def deck(t):
        p = tmp_path / ("deck_%s.txt" % t)
        p.write_text("\n".join(("t_list = " + t) if l.strip().startswith("t_list") else
                                ("dt_out = 0" if l.strip().startswith("dt_out") else l) for l in text) + "\n")
        return str(p)
    r = subprocess.run([ref, "-bfile", deck("0.05"), "-out", str(tmp_path / "start"), "-double"], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0
    start = str(tmp_path / "start" / [f for f in os.listdir(tmp_path / "start") if f.endswith(".hdr")][0])
    r1 = subprocess.run([sys.executable, "-m", "multiblockmomentsfv_b200", "-bfile", deck("0.1"), "-out",
                         str(tmp_path / "cli"), "-double", "-sfile", start], capture_output=True, text=True,
                        timeout=600, cwd=os.path.join(H.HERE, ".."))
    assert r1.returncode == 0, r1.stderr[-2000:]
    r2 = subprocess.run([ref, "-bfile", deck("0.1"), "-out", str(tmp_path / "ref"), "-double", "-sfile", start],
                        env=env, capture_output=True, text=True, timeout=600)
    assert r2.returncode == 0
    got = [f for f in os.listdir(tmp_path / "cli") if f.endswith(".hdr")]
    assert got == [f for f in os.listdir(tmp_path / "ref") if f.endswith(".hdr")]
    ok, mx, msg = output.compare(str(tmp_path / "cli" / got[0]), str(tmp_path / "ref" / got[0]), 0.0, 0.0)
    assert ok and mx == 0.0, msg


def test_bulk_copy_wait_that_runs_out_stops_the_case(monkeypatch):
    """Failure detection of the bulk tensor copies (MBM_TMA=1): every wait on a copy's
    mbarrier is bounded.  A test hook (MBM_TMA_TEST_DROP=1, one launch only) makes one warp
    withhold its first copy, so that its wait runs out: the warp flags the case and stops,
    the controller stops the case before accepting the attempt, and the call returns
    MBM_ETIMEOUT with DATA untouched.  The context stays usable: the next call runs and
    gives the bits of a run without the hook."""
    monkeypatch.setenv("MBM_TMA", "1")
    monkeypatch.setenv("MBM_AUTOTUNE", "0")       # no tuning launches before the step loop
    d = H.quadrant_deck(64, Kn=0.01, limiter=4)
    scn = sc.Scenario.seeded_quadrant(9)
    with sv.Solver(d, scn, mode="fast", show_every=0) as clean:
        clean.initialise()
        ref = clean.steps(0.0, 0.02)
        ref_layers = [clean.download(sv.L_DATA, b) for b in range(len(d.blocks))]
    monkeypatch.setenv("MBM_TMA_TEST_DROP", "1")
    with sv.Solver(d, scn, mode="fast", show_every=0) as s:
        assert s.bulk_copies()
        s.initialise()
        start = [s.download(sv.L_DATA, b) for b in range(len(d.blocks))]
        with pytest.raises(_abi.MBMError) as e:
            s.steps(0.0, 0.02)
        assert e.value.status == _abi.MBM_ETIMEOUT
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(sv.L_DATA, b), start[b], f"block {b + 1} after the stopped attempt")
        s.initialise()
        assert s.steps(0.0, 0.02) == ref
        for b in range(len(d.blocks)):
            H.assert_bitwise(s.download(sv.L_DATA, b), ref_layers[b], f"block {b + 1}")
