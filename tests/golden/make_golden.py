"""Regenerate the committed fixtures of tests/golden/ from the reference checkout.

Run from the repository root, where the reference sources are present:

    python tests/golden/make_golden.py [REFERENCE_ROOT]

Writes
  decks/*.txt             the reference's input decks (cases/*.txt), verbatim
  squareSmall_ref.npz     every zone of reference/squareSmall.ref.{hdr,dat}
                          (Float32 payload, 7 output times, Riemann2D state)
  square4_ref_t0p3.npz    the t = 0.3 zones of reference/square4.ref.{hdr,dat}
  square4_ref_trace.json  the progress lines of reference/square4.ref.txt
                          (step, CFL, time, next dt every 20 steps; steps per interval)
"""
from __future__ import annotations

import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from multiblockmomentsfv_b200 import output as out   # noqa: E402


def pack(zones, keep):
    z = [z for z in zones if keep(z)]
    return dict(
        block=np.array([q["block"] for q in z], dtype=np.int32),
        I=np.array([q["I"] for q in z], dtype=np.int32),
        J=np.array([q["J"] for q in z], dtype=np.int32),
        time=np.array([q["time"] for q in z]),
        strand=np.array([q["strand"] for q in z], dtype=np.int32),
        values=np.concatenate([q["values"].astype(np.float32).ravel() for q in z]),
    )


def main(ref_root: str = os.environ.get("MBM_REFERENCE_ROOT", "/root/reference")) -> None:
    os.makedirs(os.path.join(HERE, "decks"), exist_ok=True)
    for f in sorted(os.listdir(os.path.join(ref_root, "cases"))):
        shutil.copyfile(os.path.join(ref_root, "cases", f), os.path.join(HERE, "decks", f))

    zones, prec = out.read(os.path.join(ref_root, "reference", "squareSmall.ref"))
    assert prec == "Float32"
    np.savez_compressed(os.path.join(HERE, "squareSmall_ref.npz"), **pack(zones, lambda z: True))

    zones, prec = out.read(os.path.join(ref_root, "reference", "square4.ref"))
    np.savez_compressed(os.path.join(HERE, "square4_ref_t0p3.npz"),
                        **pack(zones, lambda z: abs(z["time"] - 0.3) < 1e-12))

    trace, intervals = [], []
    pat = re.compile(r"step:\s*(\d+)\.\.\. done\.\s+CFL: ([\d.]+), time: ([\d.]+), next dt: ([\d.]+)")
    with open(os.path.join(ref_root, "reference", "square4.ref.txt")) as f:
        for line in f:
            m = pat.search(line)
            if m:
                trace.append([len(intervals), int(m.group(1)), float(m.group(2)),
                              float(m.group(3)), float(m.group(4))])
            m = re.search(r"Append \((\d+)\)", line)
            if m:
                intervals.append(int(m.group(1)))
            m = re.search(r"Done after (\d+) steps", line)
            if m:
                total = int(m.group(1))
    with open(os.path.join(HERE, "square4_ref_trace.json"), "w") as f:
        json.dump({"records": trace, "cumulative_steps": intervals, "total_steps": total,
                   "columns": ["interval", "step", "CFL", "time", "next_dt"]}, f, indent=1)


if __name__ == "__main__":
    main(*sys.argv[1:])
