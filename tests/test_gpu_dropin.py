"""Drop-in: the reference's own C host (main, block-file parser, Mesh, Output),
linked with the GPU Steps of multiblockmomentsfv_b200/shim/mbm_steps_shim.c
(oracle/_ref/moments_b200), against the unmodified reference build
(oracle/_ref/moments) on the same decks.  Both write Float64 output (-double);
the result files must agree exactly (abstol = reltol = 0)."""
import os
import subprocess

import pytest

import helpers as H
from multiblockmomentsfv_b200 import output as out

REF = os.path.join(H.HERE, "..", "oracle", "_ref")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not os.path.exists(os.path.join(REF, "moments_b200")),
                                 reason="drop-in binary not built (make -C oracle b200)")]


def _run(exe, deck, out_dir, scenario, extra=()):
    env = dict(os.environ, MBM_SCENARIO=scenario, OMP_NUM_THREADS="1")
    r = subprocess.run([os.path.join(REF, exe), "-bfile", deck, "-out", out_dir, "-double", *extra],
                       env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hdrs = [f for f in os.listdir(out_dir) if f.endswith(".hdr")]
    assert len(hdrs) == 1
    return os.path.join(out_dir, hdrs[0]), r.stdout


def _deck(tmp_path, name, t_list=None, dt_out=None):
    text = open(os.path.join(H.DECKS, name + ".txt")).read()
    lines = []
    for line in text.splitlines():
        s = line.strip()
        if t_list is not None and s.startswith("t_list"):
            line = f"t_list = {t_list}"
        if dt_out is not None and s.startswith("dt_out"):
            line = f"dt_out = {dt_out}"
        lines.append(line)
    p = tmp_path / (name + ".txt")
    p.write_text("\n".join(lines) + "\n")
    return str(p)


@pytest.mark.parametrize("name,scenario,t_list,dt_out,extra", [
    ("squareSmall", "riemann2d", None, None, ()),
    ("square4", "riemann2d", "0.1", "0.05", ("-limiter", "superbee")),
    ("Lshape", "riemann2d", "0.02", "0.01", ("-Kn", "0.005")),
    ("ffs28", "ffs", "0.02", "0", ()),
    ("square4Box", "riemann2d", "0.05", "0", ("-R13", "1")),
    ("square4", "riemann2d", "0.1", "0.05", ("-CFL", "0.5", "-limiter", "minmod")),
])
def test_reference_host_with_gpu_steps(tmp_path, name, scenario, t_list, dt_out, extra):
    deck = _deck(tmp_path, name, t_list, dt_out)
    a, log_gpu = _run("moments_b200", deck, str(tmp_path / "gpu"), scenario, extra)
    b, _ = _run("moments", deck, str(tmp_path / "ref"), scenario, extra)
    assert os.path.basename(a) == os.path.basename(b)
    ok, mx, msg = out.compare(a, b, 0.0, 0.0)
    assert ok and mx == 0.0, msg
    ok, log = H.reference_compare(a, b, 0.0, 0.0)
    assert ok, log
    assert "(gpu)" in log_gpu or "Done after" in log_gpu


def test_reference_host_with_fast_gpu_steps(tmp_path):
    """MBM_MODE=fast in the drop-in: the reference's regression gate at its Float64
    defaults (|a - b| <= 1e-10 + 1e-8 |b|) against the unmodified reference."""
    deck = _deck(tmp_path, "square4", "0.1", "0.05")
    os.environ["MBM_MODE"] = "fast"
    try:
        a, _ = _run("moments_b200", deck, str(tmp_path / "gpu"), "riemann2d")
    finally:
        del os.environ["MBM_MODE"]
    b, _ = _run("moments", deck, str(tmp_path / "ref"), "riemann2d")
    ok, mx, msg = out.compare(a, b)
    assert ok, msg
    assert mx > 0.0          # not the bitwise kernel
    ok, log = H.reference_compare(a, b)
    assert ok, log


@pytest.mark.parametrize("mode", ["exact", "fast"])
@pytest.mark.parametrize("name", ["square4", "squareSmall"])
def test_reference_make_check(tmp_path, name, mode):
    """The reference's `make check` (Makefile:104-112) on the drop-in: the deck as
    shipped (Float32 output, every level to t = 0.3), the 2D temperature-Riemann state
    its goldens were made with, compared by tools/compare_solution.py at its default
    tolerances against reference/<deck>.ref."""
    golden = os.path.join(H.REF_BUILD, name + ".ref.hdr")
    if not os.path.exists(golden):
        pytest.skip("reference goldens not staged (make -C oracle check)")
    env = dict(os.environ, MBM_SCENARIO="riemann2d", OMP_NUM_THREADS="1", MBM_MODE=mode)
    out_dir = tmp_path / "run"
    r = subprocess.run([os.path.join(REF, "moments_b200"), "-bfile", os.path.join(H.DECKS, name + ".txt"),
                        "-out", str(out_dir)], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hdrs = [f for f in os.listdir(out_dir) if f.endswith("_tAll.hdr")]
    assert len(hdrs) == 1
    ok, log = H.reference_compare(str(out_dir / hdrs[0]), os.path.join(H.REF_BUILD, name + ".ref"))
    assert ok and log.startswith("PASS"), log


@pytest.mark.parametrize("restart_double", [True, False])
def test_reference_host_restart_with_gpu_steps(tmp_path, restart_double):
    """-sfile (src/Main.c:71-72,124): a result file written by the unmodified reference
    (squareSmall to t = 0.05, Float64 or Float32 payload) restarts both the drop-in and
    the reference, whose own LoadData (src/Mesh.c:198-283) reads it; the two runs to
    t = 0.1 must write identical files."""
    first = _deck(tmp_path, "squareSmall", "0.05", "0")
    env = dict(os.environ, MBM_SCENARIO="riemann2d", OMP_NUM_THREADS="1")
    start_dir = tmp_path / "start"
    r = subprocess.run([os.path.join(REF, "moments"), "-bfile", first, "-out", str(start_dir)]
                       + (["-double"] if restart_double else []), env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    start = [f for f in os.listdir(start_dir) if f.endswith(".hdr")][0]
    sfile = str(start_dir / start)
    deck = _deck(tmp_path, "squareSmall", "0.1", "0")
    a, log_gpu = _run("moments_b200", deck, str(tmp_path / "gpu"), "riemann2d", ("-sfile", sfile))
    b, log_ref = _run("moments", deck, str(tmp_path / "ref"), "riemann2d", ("-sfile", sfile))
    assert "Read file" in log_gpu and "Read file" in log_ref
    assert os.path.basename(a) == os.path.basename(b)
    ok, mx, msg = out.compare(a, b, 0.0, 0.0)
    assert ok and mx == 0.0, msg
    ok, log = H.reference_compare(a, b, 0.0, 0.0)
    assert ok, log
