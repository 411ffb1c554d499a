"""The CPU reference arm of bench.py (the reference's own Steps, OpenMP build in
oracle/_ref): its JSON line carries the fields the bench contract asks for, on a
bounded sample of the benchmark layout."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libmbmref_omp.so")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference build absent (oracle/_ref)")


def _last_json(out: str) -> dict:
    return json.loads(out.strip().splitlines()[-1])


def test_ref_bench_small_grid():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "oracle", "ref_bench.py"), "--n", "64", "--steps", "2",
                        "--warmup", "1", "--threads", "2"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    d = _last_json(r.stdout)
    # Steps runs to an end time set for 2 settled steps after its first, shorter one
    assert d["n"] == 64 and d["cells"] == 4 * 64 * 64 and 2 <= d["steps"] <= 4
    assert d["driver"] == "Steps"
    assert d["value"] > 0 and d["seconds"] > 0 and d["cores"] >= 1


def test_bench_reference_arm_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    d = _last_json(r.stdout)
    assert d["impl"] == "reference" and "unavailable" not in d
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["unit"] == "cell-updates/s" and d["higher_is_better"] is True and d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0
    assert d["warmup"] >= 3          # the contract's minimum, whatever was asked
